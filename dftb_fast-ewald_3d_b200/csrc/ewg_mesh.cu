// ewg_mesh.cu -- the Gaussian-window NFFT of the reciprocal sum on the GPU.
//
// Pipeline for one evaluation (reference: fft/ewald_fft_3d_fourier.f90:28-153
// and nfft/nfft.f90:196-404):
//   weights   per-atom 3 x (2m+1) window weights      (stencil_weights :122-159)
//   spread    tile-owned, deterministic, no atomics   (adjoint step 1 :253-278)
//   R2C x     real rows -> k1 in [0, M1/2]            (adjoint step 2 :282, pruned)
//   C2C y     -> k2 in [-M2/2, M2/2]
//   C2C z + influence + inverse z (fused)             (deconvolution :286-298,
//             weights :92-119, ik derivative :130-151, embedding :362-375)
//   C2C y inverse, C2R x inverse                      (forward step 2 :378)
//   gather    per-atom, 1 or 4 components             (forward step 3 :380-402)
//
// Sign conventions.  With G(k) = sum_x g(x) exp(-2 pi i k.x/n) (the standard
// forward transform of the spread grid) and Q(k) = w(k) f(k)^2 G(k), f the
// per-axis deconvolution factors, the real part the reference takes of its
// forward NFFT equals the standard inverse transform of c(k) Q(k) over the
// closed box |k_d| <= M_d/2, where c(k) = ([k in S] + [-k in S]) / 2 and S is
// the reference's mode set [-M/2, M/2-1]^3 (nfft/nfft.f90:61-75).  Only k1 >= 0
// is stored (Hermitian half).
//
// Force grids.  The reference differentiates in Fourier space along each
// Cartesian axis, -i k_c c(k) Q(k) with k_c = 2 pi sum_d k_d b_dc
// (fft/ewald_fft_3d_fourier.f90:130-151).  The same force follows from the
// three fractional derivatives D_d = d(phi)/d(s_d), spectra 2 pi i k_d c Q, as
// F = -q sum_d D_d b_d.  In that basis each multiplication by k_d commutes with
// the transforms along the other axes, so fewer transforms are needed:
//   z inverse  P = IFFT_z(cQ), T3 = IFFT_z(2 pi i k3 cQ)                    (2, not 4)
//   y inverse  Y0 = IFFT_y(P), Y2 = IFFT_y(2 pi i k2 P), Y3 = IFFT_y(T3)     (3, not 4)
//   x C2R      phi = C2R(Y0), D1 = C2R(2 pi i k1 Y0), D2 = C2R(Y2), D3 = C2R(Y3).
// The result equals the Cartesian form up to rounding.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <type_traits>

#include "ewg_fft.cuh"
#include "ewg_kernels.h"

namespace ewg {

namespace {

constexpr size_t kSmemBudget = 200 * 1024;

// Every pass transforms L lines (a power of two, the fastest index) of length n
// with fft_edges: two buffers of n * L elements in shared memory, blockDim.x =
// pass_threads(L): 32 threads per line, at least 128 per CTA.  The first and
// last radix passes read and write global memory directly.
constexpr int pass_threads(int L) { return L >= 4 ? 32 * L : 128; }

// The buffer the last pass of `plan` leaves free (its `spare`).
template <typename R>
__device__ __forceinline__ cx<R>* spare_buffer(cx<R>* a, cx<R>* b, const FftPlan& plan) {
  return (plan.nstages & 1) ? a : b;
}

// Transform shapes: the generic runtime schedule, or a length and three-radix
// schedule fixed at compile time (fft_static3) for the lengths the benchmark
// configurations use most.
struct DynShape {
  template <int L>
  static constexpr int threads() { return pass_threads(L); }
  template <typename R, int SIGN, int L, class Ld, class St>
  __device__ __forceinline__ static void run(cx<R>* a, cx<R>* b, int n, const FftPlan& plan,
                                             const cx<R>* __restrict__ tw, Ld ld, St st) {
    fft_edges<R, SIGN, L>(a, b, n, plan, tw, ld, st);
  }
};
// TPL threads per line: the butterflies of a pass per line are N / radix, so a
// count that divides them (or just exceeds them) saves rounds over 32.
template <int N, int R0, int R1, int R2, int TPL = 32>
struct StatShape {
  template <int L>
  static constexpr int threads() { return L * TPL; }
  template <typename R, int SIGN, int L, class Ld, class St>
  __device__ __forceinline__ static void run(cx<R>* a, cx<R>* b, int, const FftPlan&,
                                             const cx<R>* __restrict__ tw, Ld ld, St st) {
    fft_static3<R, SIGN, L, L * TPL, N, R0, R1, R2>(a, b, tw, ld, st);
  }
};

// ---------------------------------------------------------------------------
// x pass, real to complex: row pairs (2p, 2p+1) form one complex line; keep
// k1 = 0..K1-1 of each row.
// ---------------------------------------------------------------------------
template <typename R, int L, class SH>
__device__ __forceinline__ void fft_x_r2c_body(int bx, const R* __restrict__ grid,
                                                               cx<R>* __restrict__ A1, int n1,
                                                               int npairs, int K1, FftPlan plan) {
  chain_enter();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<R>* a = reinterpret_cast<cx<R>*>(smem_raw);
  cx<R>* b = a + static_cast<size_t>(n1) * L;
  const cx<R>* tw = plan_twiddles<R>(plan);
  const int pair0 = bx * L;
  // Each thread serves one line (its lane in the group): resolve its rows once.
  const bool valid = pair0 + static_cast<int>(threadIdx.x & (L - 1)) < npairs;
  const R* ra = grid + static_cast<size_t>(2 * (pair0 + (threadIdx.x & (L - 1)))) * n1;
  const R* rb = ra + n1;
  auto load = [&](int, int x) { return valid ? mk(ra[x], rb[x]) : mk(R(0), R(0)); };
  auto store = [&](int l, int k, cx<R> v, cx<R>* spare) { spare[k * L + l] = v; };
  SH::template run<R, -1, L>(a, b, n1, plan, tw, load, store);
  __syncthreads();
  const cx<R>* res = spare_buffer(a, b, plan);
  const R h = R(0.5);
  for (int t = threadIdx.x; t < K1 * L; t += blockDim.x) {
    const int l = t % L, k = t / L;  // L is a power of two
    const int pr = pair0 + l;
    if (pr >= npairs) continue;
    const cx<R> z = res[k * L + l];
    cx<R> zc = res[(k == 0 ? 0 : n1 - k) * L + l];
    zc.y = -zc.y;
    const size_t row = static_cast<size_t>(2 * pr);
    A1[row * K1 + k] = mk(h * (z.x + zc.x), h * (z.y + zc.y));
    A1[(row + 1) * K1 + k] = mk(h * (z.y - zc.y), -h * (z.x - zc.x));
  }
}

// ---------------------------------------------------------------------------
// y pass, forward: lines over i2 for (i3, k1-block); keep k2 in [-H2, H2].
// ---------------------------------------------------------------------------
template <typename R, int L, class SH>
__device__ __forceinline__ void fft_y_fwd_body(int bx, int by, const cx<R>* __restrict__ A1,
                                                               cx<R>* __restrict__ A2, int n2,
                                                               int K1, int K2, int H2,
                                                               FftPlan plan) {
  chain_enter();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<R>* a = reinterpret_cast<cx<R>*>(smem_raw);
  cx<R>* b = a + static_cast<size_t>(n2) * L;
  const cx<R>* tw = plan_twiddles<R>(plan);
  const int k0 = bx * L;
  const int i3 = by;
  const int kl = k0 + static_cast<int>(threadIdx.x & (L - 1));  // this thread's k1
  const bool kin = kl < K1;
  const cx<R>* src = A1 + static_cast<size_t>(i3) * n2 * K1 + kl;
  cx<R>* dst = A2 + static_cast<size_t>(i3) * K2 * K1 + kl;
  auto load = [&](int, int i2) { return kin ? src[i2 * K1] : mk(R(0), R(0)); };
  auto store = [&](int, int e, cx<R> v, cx<R>*) {
    int k2i;
    if (e <= H2)
      k2i = e + H2;
    else if (e >= n2 - H2)
      k2i = e - n2 + H2;
    else
      return;
    if (kin) dst[k2i * K1] = v;
  };
  SH::template run<R, -1, L>(a, b, n2, plan, tw, load, store);
}

// ---------------------------------------------------------------------------
// z pass forward, influence weights, z pass inverse -- fused per (k2, k1-block).
// ---------------------------------------------------------------------------
struct InfluenceArgs {
  int H[3];            // closed box |k_d| <= H_d
  int slo[3], shi[3];  // mode set S_d = [slo_d, shi_d] (nfft/nfft.f90:61-75)
  double rec[3][3];
  double prefactor;    // 4 pi / V
  double inv4a2;       // 1 / (4 alpha^2)
  const double* corr2[3];
  // Optional: per-CTA partial of the reciprocal strain derivative dE_k/d eps
  // (xx, yy, zz, xy, xz, yz), 6 doubles at (blockIdx.y * gridDim.x + blockIdx.x) * 6.
  double* stress;
};

// nz = 1 (potential) or 2 (also T3, the spectrum times 2 pi i k3).
template <typename R, int L, bool STRESS, class SH>
__device__ __forceinline__ void fft_z_influence_body(
    int bx, int by, int gx, const cx<R>* __restrict__ A2, cx<R>* __restrict__ B2, int n3, int K1, int K2, int K3, int nz,
    InfluenceArgs ia, FftPlan plan) {
  chain_enter();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<R>* a = reinterpret_cast<cx<R>*>(smem_raw);
  cx<R>* b = a + static_cast<size_t>(n3) * L;
  cx<R>* q = b + static_cast<size_t>(n3) * L;  // K3 weighted modes per line
  const cx<R>* tw = plan_twiddles<R>(plan);
  const int k0 = bx * L;
  const int k2i = by;
  const int h1 = ia.H[0], h2 = ia.H[1], h3 = ia.H[2];
  const int k2 = k2i - h2;
  const double twoPi = 2.0 * 3.14159265358979323846;
  const int kl = k0 + static_cast<int>(threadIdx.x & (L - 1));  // this thread's k1
  const bool kin = kl < K1;
  const size_t zstride = static_cast<size_t>(K2) * K1;
  const cx<R>* src = A2 + static_cast<size_t>(k2i) * K1 + kl;
  auto load_fwd = [&](int, int i3) { return kin ? src[i3 * zstride] : mk(R(0), R(0)); };
  // Reciprocal strain derivative of E_k = sum_k 1/2 w(k) |G(k)|^2 (w with the
  // deconvolution f^2 and the Nyquist factor c(k)): under a homogeneous strain
  // k -> (1 - eps) k and V -> V (1 + tr eps), so each mode adds
  // 1/2 w |G|^2 (2 k_a k_b (1/(4 alpha^2) + 1/k^2) - delta_ab); modes with k1 > 0
  // stand for the pair (k, -k).
  double sv[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  // Weight each mode of the closed box as it leaves the forward transform.
  auto store_weighted = [&](int l, int e, cx<R> g, cx<R>*) {
    int k3;
    if (e <= h3)
      k3 = e;
    else if (e >= n3 - h3)
      k3 = e - n3;
    else
      return;
    const int k1 = k0 + l;
    double wt = 0.0;
    if (k1 < K1 && !(k1 == 0 && k2 == 0 && k3 == 0)) {
      double kv[3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
        kv[c] = twoPi * (k1 * ia.rec[0][c] + k2 * ia.rec[1][c] + k3 * ia.rec[2][c]);
      const double kk2 = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
      if (kk2 >= 1.0e-24) {
        const int inS = (k1 >= ia.slo[0] && k1 <= ia.shi[0]) && (k2 >= ia.slo[1] && k2 <= ia.shi[1]) &&
                        (k3 >= ia.slo[2] && k3 <= ia.shi[2]);
        const int inMinusS = (-k1 >= ia.slo[0] && -k1 <= ia.shi[0]) &&
                             (-k2 >= ia.slo[1] && -k2 <= ia.shi[1]) &&
                             (-k3 >= ia.slo[2] && -k3 <= ia.shi[2]);
        const double cw = 0.5 * (inS + inMinusS);
        wt = cw * ia.prefactor * exp(-kk2 * ia.inv4a2) / kk2 * ia.corr2[0][k1 + h1] *
             ia.corr2[1][k2 + h2] * ia.corr2[2][k3 + h3];
        if constexpr (STRESS) {
          const double gx = static_cast<double>(g.x), gy = static_cast<double>(g.y);
          const double e = (k1 > 0 ? 1.0 : 0.5) * wt * (gx * gx + gy * gy);
          const double f = 2.0 * (ia.inv4a2 + 1.0 / kk2);
          sv[0] += e * (f * kv[0] * kv[0] - 1.0);
          sv[1] += e * (f * kv[1] * kv[1] - 1.0);
          sv[2] += e * (f * kv[2] * kv[2] - 1.0);
          sv[3] += e * f * kv[0] * kv[1];
          sv[4] += e * f * kv[0] * kv[2];
          sv[5] += e * f * kv[1] * kv[2];
        }
      }
    }
    q[(k3 + h3) * L + l] = mk(static_cast<R>(wt * static_cast<double>(g.x)),
                              static_cast<R>(wt * static_cast<double>(g.y)));
  };
  SH::template run<R, -1, L>(a, b, n3, plan, tw, load_fwd, store_weighted);
  __syncthreads();
  if constexpr (STRESS) {  // fixed-order CTA sum: shuffle tree per warp, then warps in order
    __shared__ double sred[32][6];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) sv[j] += __shfl_xor_sync(0xffffffffu, sv[j], off);
      if (lane == 0) sred[warp][j] = sv[j];
    }
    __syncthreads();
    if (threadIdx.x < 6) {
      double t = 0.0;
      for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += sred[w][threadIdx.x];
      ia.stress[(static_cast<size_t>(by) * gx + bx) * 6 + threadIdx.x] = t;
    }
  }
  for (int c = 0; c < nz; ++c) {
    auto load_inv = [&](int l, int i3) {
      int k3;
      if (i3 <= h3)
        k3 = i3;
      else if (i3 >= n3 - h3)
        k3 = i3 - n3;
      else
        return mk(R(0), R(0));
      cx<R> v = q[(k3 + h3) * L + l];
      if (c > 0) {
        const R t = static_cast<R>(twoPi * k3);
        v = mk(-t * v.y, t * v.x);  // 2 pi i k3 v
      }
      return v;
    };
    cx<R>* dst = B2 + static_cast<size_t>(c) * n3 * zstride + static_cast<size_t>(k2i) * K1 + kl;
    auto store = [&](int, int i3, cx<R> v, cx<R>*) {
      if (kin) dst[i3 * zstride] = v;
    };
    SH::template run<R, 1, L>(a, b, n3, plan, tw, load_inv, store);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// y pass inverse: zero-padded k2 box -> i2, for (k1-block, i3, component).
// Components: 0 = IFFT_y(P) and, for forces, 1 = IFFT_y(2 pi i k2 P),
// 2 = IFFT_y(T3), with P and T3 the z pass's two outputs.
// ---------------------------------------------------------------------------
template <typename R, int L, class SH>
__device__ __forceinline__ void fft_y_inv_body(int bx, int by, int bz, const cx<R>* __restrict__ B2,
                                                               cx<R>* __restrict__ B1, int n2,
                                                               int n3, int K1, int K2, int H2,
                                                               FftPlan plan) {
  chain_enter();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<R>* a = reinterpret_cast<cx<R>*>(smem_raw);
  cx<R>* b = a + static_cast<size_t>(n2) * L;
  const cx<R>* tw = plan_twiddles<R>(plan);
  const int k0 = bx * L;
  const int i3 = by;
  const int c = bz;
  const int cs = c == 2 ? 1 : 0;  // source component in B2
  const bool dk2 = c == 1;        // times 2 pi i k2
  const int kl = k0 + static_cast<int>(threadIdx.x & (L - 1));  // this thread's k1
  const bool kin = kl < K1;
  // src points at the k2 = 0 row of this line's (i3, k1) column.
  const cx<R>* src = B2 + ((static_cast<size_t>(cs) * n3 + i3) * K2 + H2) * K1 + kl;
  cx<R>* dst = B1 + (static_cast<size_t>(c) * n3 + i3) * n2 * K1 + kl;
  auto load = [&](int, int i2) {
    int k2;
    if (i2 <= H2)
      k2 = i2;
    else if (i2 >= n2 - H2)
      k2 = i2 - n2;
    else
      return mk(R(0), R(0));
    cx<R> v = kin ? src[k2 * K1] : mk(R(0), R(0));
    if (dk2) {
      const R t = static_cast<R>(2.0 * 3.14159265358979323846 * k2);
      v = mk(-t * v.y, t * v.x);
    }
    return v;
  };
  auto store = [&](int, int i2, cx<R> v, cx<R>*) {
    if (kin) dst[i2 * K1] = v;
  };
  SH::template run<R, 1, L>(a, b, n2, plan, tw, load, store);
}

// ---------------------------------------------------------------------------
// x pass, complex to real.  Lines are (row pair, component) with the component
// fastest: line = l * NCG + cc, NP = L / NCG pairs and NCG components per CTA,
// so neighbouring threads write the components of one grid point; output
// interleaved with nc components per grid point.  With nc = 4 the outputs are
// phi = C2R(Y0), D1 = C2R(2 pi i k1 Y0), D2 = C2R(Y2), D3 = C2R(Y3), Y0, Y2, Y3
// the y pass's three components.
// ---------------------------------------------------------------------------
template <typename R, int L, int NCG, class SH>
__device__ __forceinline__ void fft_x_c2r_body(int bx, int by, const cx<R>* __restrict__ B1,
                                                               R* __restrict__ out, int n1,
                                                               int nrows, int K1, int nc,
                                                               FftPlan plan) {
  chain_enter();
  constexpr int NP = L / NCG;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<R>* a = reinterpret_cast<cx<R>*>(smem_raw);
  cx<R>* b = a + static_cast<size_t>(n1) * L;
  const cx<R>* tw = plan_twiddles<R>(plan);
  const int pair0 = bx * NP;
  const int c0 = by * NCG;
  const int npairs = nrows / 2;
  // Each thread serves one line: resolve its rows and output columns once.
  const int line = static_cast<int>(threadIdx.x & (L - 1));
  const int cc = line % NCG, pr = pair0 + line / NCG;
  const bool valid = pr < npairs;
  const int co = c0 + cc;               // output component
  const int cs = co <= 1 ? 0 : co - 1;  // its source component in B1
  const bool dk1 = co == 1;             // times 2 pi i k1
  const cx<R>* sa = B1 + (static_cast<size_t>(cs) * nrows + 2 * static_cast<size_t>(pr)) * K1;
  const cx<R>* sb = sa + K1;
  R* oa = out + 2 * static_cast<size_t>(pr) * n1 * nc + c0 + cc;
  R* ob = oa + static_cast<size_t>(n1) * nc;
  auto load = [&](int, int x) {
    const bool lo = x < K1;
    const bool hi = x > n1 - K1;
    cx<R> fa = mk(R(0), R(0)), fb = mk(R(0), R(0));
    if (valid && (lo || hi)) {
      const int kx = lo ? x : n1 - x;
      fa = sa[kx];
      fb = sb[kx];
      if (dk1) {
        const R t = static_cast<R>(2.0 * 3.14159265358979323846 * kx);
        fa = mk(-t * fa.y, t * fa.x);
        fb = mk(-t * fb.y, t * fb.x);
      }
      if (x == 0) {
        fa.y = R(0);
        fb.y = R(0);
      } else if (hi) {
        fa.y = -fa.y;
        fb.y = -fb.y;
      }
    }
    return mk(fa.x - fb.y, fa.y + fb.x);
  };
  auto store = [&](int, int x, cx<R> v, cx<R>*) {
    if (!valid) return;
    oa[x * nc] = v.x;
    ob[x * nc] = v.y;
  };
  SH::template run<R, 1, L>(a, b, n1, plan, tw, load, store);
}

// ---- pass kernels: one cell (blockIdx = the pass's block), or every cell of a
// batch (blockIdx.x over the cells' blocks end to end; the cell's lengths,
// plans and buffers from the batch table; the lines per CTA are common).
template <typename R, int L, class SH = DynShape>
__global__ void __launch_bounds__(SH::template threads<L>()) k_fft_x_r2c(const R* __restrict__ grid,
                                                               cx<R>* __restrict__ A1, int n1,
                                                               int npairs, int K1, FftPlan plan) {
  fft_x_r2c_body<R, L, SH>(blockIdx.x, grid, A1, n1, npairs, K1, plan);
}
template <typename R, int L, class SH = DynShape>
__global__ void __launch_bounds__(SH::template threads<L>()) k_fft_y_fwd(const cx<R>* __restrict__ A1,
                                                               cx<R>* __restrict__ A2, int n2,
                                                               int K1, int K2, int H2,
                                                               FftPlan plan) {
  fft_y_fwd_body<R, L, SH>(blockIdx.x, blockIdx.y, A1, A2, n2, K1, K2, H2, plan);
}
template <typename R, int L, bool STRESS, class SH = DynShape>
__global__ void __launch_bounds__(SH::template threads<L>()) k_fft_z_influence(
    const cx<R>* __restrict__ A2, cx<R>* __restrict__ B2, int n3, int K1, int K2, int K3, int nz,
    InfluenceArgs ia, FftPlan plan) {
  fft_z_influence_body<R, L, STRESS, SH>(blockIdx.x, blockIdx.y, gridDim.x, A2, B2, n3, K1, K2,
                                         K3, nz, ia, plan);
}
template <typename R, int L, class SH = DynShape>
__global__ void __launch_bounds__(SH::template threads<L>()) k_fft_y_inv(const cx<R>* __restrict__ B2,
                                                               cx<R>* __restrict__ B1, int n2,
                                                               int n3, int K1, int K2, int H2,
                                                               FftPlan plan) {
  fft_y_inv_body<R, L, SH>(blockIdx.x, blockIdx.y, blockIdx.z, B2, B1, n2, n3, K1, K2, H2, plan);
}
template <typename R, int L, int NCG, class SH = DynShape>
__global__ void __launch_bounds__(SH::template threads<L>()) k_fft_x_c2r(const cx<R>* __restrict__ B1,
                                                               R* __restrict__ out, int n1,
                                                               int nrows, int K1, int nc,
                                                               FftPlan plan) {
  fft_x_c2r_body<R, L, NCG, SH>(blockIdx.x, blockIdx.y, B1, out, n1, nrows, K1, nc, plan);
}

// Blocks per cell of each pass (r2c, y forward, z, y inverse, c2r) at L lines
// per CTA, nc grids through the inverse passes.
__host__ __device__ inline void pass_blocks(const MeshGeom& g, int L, int nc, int out[5]) {
  const int npairs = g.n[1] * g.n[2] / 2, kb = (g.K1 + L - 1) / L;
  out[0] = (npairs + L - 1) / L;
  out[1] = kb * g.n[2];
  out[2] = kb * g.K2;
  out[3] = kb * g.n[2] * (nc == 4 ? 3 : 1);
  out[4] = (nc == 4 && L >= 4) ? (npairs + L / 4 - 1) / (L / 4) : ((npairs + L - 1) / L) * nc;
}

__device__ __forceinline__ const BatchCell& pass_cell(const BatchCell* __restrict__ cells,
                                                      const int* __restrict__ prefix, int ncells,
                                                      int* local) {
  const int c = seg_cell(prefix, ncells, blockIdx.x);
  *local = static_cast<int>(blockIdx.x) - prefix[c];
  return cells[c];
}

template <typename R, int L, class SH = DynShape>
__global__ void __launch_bounds__(SH::template threads<L>()) k_fft_x_r2c_seg(
    const BatchCell* __restrict__ cells, const int* __restrict__ prefix, int ncells) {
  int local;
  const BatchCell& bc = pass_cell(cells, prefix, ncells, &local);
  const FftPlan plan = bc.fft[0];
  fft_x_r2c_body<R, L, SH>(local, static_cast<const R*>(bc.grid), static_cast<cx<R>*>(bc.A1),
                       bc.g.n[0], bc.g.n[1] * bc.g.n[2] / 2, bc.g.K1, plan);
}
template <typename R, int L, class SH = DynShape>
__global__ void __launch_bounds__(SH::template threads<L>()) k_fft_y_fwd_seg(
    const BatchCell* __restrict__ cells, const int* __restrict__ prefix, int ncells) {
  int local;
  const BatchCell& bc = pass_cell(cells, prefix, ncells, &local);
  const int kb = (bc.g.K1 + L - 1) / L;
  const FftPlan plan = bc.fft[1];
  fft_y_fwd_body<R, L, SH>(local % kb, local / kb, static_cast<const cx<R>*>(bc.A1),
                       static_cast<cx<R>*>(bc.A2), bc.g.n[1], bc.g.K1, bc.g.K2,
                       (bc.g.K2 - 1) / 2, plan);
}
template <typename R, int L, class SH = DynShape>
__global__ void __launch_bounds__(SH::template threads<L>()) k_fft_z_influence_seg(
    const BatchCell* __restrict__ cells, const int* __restrict__ prefix, int ncells, int nz) {
  int local;
  const BatchCell& bc = pass_cell(cells, prefix, ncells, &local);
  const int kb = (bc.g.K1 + L - 1) / L;
  InfluenceArgs ia;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    ia.H[d] = bc.g.M[d] - bc.g.M[d] / 2;
    ia.slo[d] = bc.g.M[d] / 2 - bc.g.M[d];
    ia.shi[d] = bc.g.M[d] / 2 - 1;
    ia.corr2[d] = bc.corr2[d];
#pragma unroll
    for (int e = 0; e < 3; ++e) ia.rec[d][e] = bc.g.rec[d][e];
  }
  ia.prefactor = 4.0 * 3.14159265358979323846 / bc.g.volume;
  ia.inv4a2 = 1.0 / (4.0 * (bc.g.alpha * bc.g.alpha));
  ia.stress = nullptr;
  const FftPlan plan = bc.fft[2];
  fft_z_influence_body<R, L, false, SH>(local % kb, local / kb, kb, static_cast<const cx<R>*>(bc.A2),
                                    static_cast<cx<R>*>(bc.B2), bc.g.n[2], bc.g.K1, bc.g.K2,
                                    bc.g.K3, nz, ia, plan);
}
template <typename R, int L, class SH = DynShape>
__global__ void __launch_bounds__(SH::template threads<L>()) k_fft_y_inv_seg(
    const BatchCell* __restrict__ cells, const int* __restrict__ prefix, int ncells) {
  int local;
  const BatchCell& bc = pass_cell(cells, prefix, ncells, &local);
  const int kb = (bc.g.K1 + L - 1) / L, n3 = bc.g.n[2];
  const int t = local / kb;
  const FftPlan plan = bc.fft[1];
  fft_y_inv_body<R, L, SH>(local % kb, t % n3, t / n3, static_cast<const cx<R>*>(bc.B2),
                       static_cast<cx<R>*>(bc.B1), bc.g.n[1], n3, bc.g.K1, bc.g.K2,
                       (bc.g.K2 - 1) / 2, plan);
}
template <typename R, int L, int NCG, class SH = DynShape>
__global__ void __launch_bounds__(SH::template threads<L>()) k_fft_x_c2r_seg(
    const BatchCell* __restrict__ cells, const int* __restrict__ prefix, int ncells, int nc) {
  int local;
  const BatchCell& bc = pass_cell(cells, prefix, ncells, &local);
  const int nrows = bc.g.n[1] * bc.g.n[2];
  const int nbx = (nrows / 2 + L / NCG - 1) / (L / NCG);
  const FftPlan plan = bc.fft[0];
  fft_x_c2r_body<R, L, NCG, SH>(local % nbx, local / nbx, static_cast<const cx<R>*>(bc.B1),
                            static_cast<R*>(bc.out), bc.g.n[0], nrows, bc.g.K1, nc, plan);
}

template <typename R>
size_t cbytes() {
  return sizeof(cx<R>);
}

// Shared bytes of one pass CTA: two ping-pong buffers of L lines plus `extra`
// elements per line.
size_t pass_smem(int n, int L, size_t cb, int extra) {
  return (2 * static_cast<size_t>(n) + extra) * L * cb;
}

// Lines per CTA: 8 when that fits in 64 KB (several CTAs per SM), else the
// largest of 4, 2, 1 within the per-CTA budget; 0 when even one line does not fit.
int pick_lines(int n, size_t cb, int extra = 0) {
  if (pass_smem(n, 8, cb, extra) <= 64 * 1024) return 8;
  for (int L = 4; L >= 1; L /= 2)
    if (pass_smem(n, L, cb, extra) <= kSmemBudget) return L;
  return 0;
}

// Lines per CTA of one single-cell pass: pick_lines, capped by the plan's
// kernel shape (the cap only lowers L, so the buffers still fit).
int plan_lines(const MeshPlan& mp, int n, size_t cb, int extra = 0) {
  const int L = pick_lines(n, cb, extra);
  return mp.lines_cap > 0 && mp.lines_cap < L ? mp.lines_cap : L;
}

// Calls f(std::integral_constant<int, L>) for L in {1, 2, 4, 8}.
template <typename F>
void with_lines(int L, F&& f) {
  switch (L) {
    case 8: f(std::integral_constant<int, 8>{}); break;
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 2: f(std::integral_constant<int, 2>{}); break;
    default: f(std::integral_constant<int, 1>{}); break;
  }
}

// Calls f(shape) with the compile-time shape of the plan's length when one is
// specialised for this precision and lines per CTA (and the plan's radix
// schedule is the one specialised), else f(DynShape{}).
template <int N, int R0, int R1, int R2>
bool is_schedule(const FftPlan& p) {
  return p.n == N && p.nstages == 3 && p.radix[0] == R0 && p.radix[1] == R1 && p.radix[2] == R2;
}
template <typename R, int L, typename F>
void with_shape(const FftPlan& p, F&& f) {
  if constexpr (sizeof(R) == 8 && L == 4) {
    if (is_schedule<280, 7, 5, 8>(p)) return f(StatShape<280, 7, 5, 8, 40>{});
    if (is_schedule<512, 8, 8, 8>(p)) return f(StatShape<512, 8, 8, 8, 64>{});
  }
  if constexpr (sizeof(R) == 8 && L == 8) {
    if (is_schedule<128, 8, 8, 2>(p)) return f(StatShape<128, 8, 8, 2>{});
  }
  if constexpr (sizeof(R) == 4 && L == 8) {
    if (is_schedule<140, 7, 5, 4>(p)) return f(StatShape<140, 7, 5, 4, 36>{});
    if (is_schedule<160, 5, 8, 4>(p)) return f(StatShape<160, 5, 8, 4, 40>{});
    if (is_schedule<280, 7, 5, 8>(p)) return f(StatShape<280, 7, 5, 8, 40>{});
  }
  f(DynShape{});
}

template <typename R>
void forward_impl(const MeshPlan& mp, const void* grid, void* A1v, void* A2v, void* B2v, int nc,
                  double* stress_part, cudaStream_t st) {
  const MeshGeom& g = mp.g;
  const int n1 = g.n[0], n2 = g.n[1], n3 = g.n[2];
  cx<R>* A1 = static_cast<cx<R>*>(A1v);
  cx<R>* A2 = static_cast<cx<R>*>(A2v);
  cx<R>* B2 = static_cast<cx<R>*>(B2v);
  const size_t cb = cbytes<R>();
  {  // x, real to complex
    prof_mark(mp.prof, st, ST_FFT_X_R2C);
    const int npairs = n2 * n3 / 2;
    const int L = plan_lines(mp, n1, cb);
    const size_t sm = pass_smem(n1, L, cb, 0);
    const int blocks = (npairs + L - 1) / L;
    with_lines(L, [&](auto lc) {
      constexpr int LL = decltype(lc)::value;
      with_shape<R, LL>(mp.fft[0], [&](auto sh) {
        launch_chained(k_fft_x_r2c<R, LL, decltype(sh)>, blocks, decltype(sh)::template threads<LL>(), sm, st,
                       static_cast<const R*>(grid), A1, n1, npairs, g.K1, mp.fft[0]);
      });
    });
    ++g_launches;
  }
  {  // y forward
    prof_mark(mp.prof, st, ST_FFT_Y_FWD);
    const int L = plan_lines(mp, n2, cb);
    const size_t sm = pass_smem(n2, L, cb, 0);
    dim3 grd((g.K1 + L - 1) / L, n3);
    const int H2 = (g.K2 - 1) / 2;
    with_lines(L, [&](auto lc) {
      constexpr int LL = decltype(lc)::value;
      with_shape<R, LL>(mp.fft[1], [&](auto sh) {
        launch_chained(k_fft_y_fwd<R, LL, decltype(sh)>, grd, decltype(sh)::template threads<LL>(), sm, st, A1, A2, n2,
                       g.K1, g.K2, H2, mp.fft[1]);
      });
    });
    ++g_launches;
  }
  {  // z forward + influence + z inverse
    prof_mark(mp.prof, st, ST_FFT_Z_INFL);
    const int nz = nc == 4 ? 2 : 1;
    InfluenceArgs ia;
    for (int d = 0; d < 3; ++d) {
      ia.H[d] = g.M[d] - g.M[d] / 2;
      ia.slo[d] = g.M[d] / 2 - g.M[d];
      ia.shi[d] = g.M[d] / 2 - 1;
    }
    for (int i = 0; i < 3; ++i)
      for (int d = 0; d < 3; ++d) ia.rec[i][d] = g.rec[i][d];
    ia.prefactor = 4.0 * kPi / g.volume;
    ia.inv4a2 = 1.0 / (4.0 * (g.alpha * g.alpha));
    for (int d = 0; d < 3; ++d) ia.corr2[d] = mp.corr2[d];
    ia.stress = stress_part;
    const int L = plan_lines(mp, n3, cb, g.K3);
    const size_t sm = pass_smem(n3, L, cb, g.K3);
    dim3 grd((g.K1 + L - 1) / L, g.K2);
    with_lines(L, [&](auto lc) {
      constexpr int LL = decltype(lc)::value;
      with_shape<R, LL>(mp.fft[2], [&](auto sh) {
        using SH = decltype(sh);
        if (stress_part)
          launch_chained(k_fft_z_influence<R, LL, true, SH>, grd, SH::template threads<LL>(), sm, st, A2, B2,
                         n3, g.K1, g.K2, g.K3, nz, ia, mp.fft[2]);
        else
          launch_chained(k_fft_z_influence<R, LL, false, SH>, grd, SH::template threads<LL>(), sm, st, A2, B2,
                         n3, g.K1, g.K2, g.K3, nz, ia, mp.fft[2]);
      });
    });
    ++g_launches;
  }
}

template <typename R>
void inverse_impl(const MeshPlan& mp, const void* B2v, void* B1v, void* out, int nc,
                  cudaStream_t st) {
  const MeshGeom& g = mp.g;
  const int n1 = g.n[0], n2 = g.n[1], n3 = g.n[2];
  const cx<R>* B2 = static_cast<const cx<R>*>(B2v);
  cx<R>* B1 = static_cast<cx<R>*>(B1v);
  const size_t cb = cbytes<R>();
  {
    prof_mark(mp.prof, st, ST_FFT_Y_INV);
    const int L = plan_lines(mp, n2, cb);
    const size_t sm = pass_smem(n2, L, cb, 0);
    dim3 grd((g.K1 + L - 1) / L, n3, nc == 4 ? 3 : 1);
    const int H2 = (g.K2 - 1) / 2;
    with_lines(L, [&](auto lc) {
      constexpr int LL = decltype(lc)::value;
      with_shape<R, LL>(mp.fft[1], [&](auto sh) {
        launch_chained(k_fft_y_inv<R, LL, decltype(sh)>, grd, decltype(sh)::template threads<LL>(), sm, st, B2, B1, n2,
                       n3, g.K1, g.K2, H2, mp.fft[1]);
      });
    });
    ++g_launches;
  }
  {
    prof_mark(mp.prof, st, ST_FFT_X_C2R);
    const int nrows = n2 * n3;
    const int L = plan_lines(mp, n1, cb);
    const size_t sm = pass_smem(n1, L, cb, 0);
    R* o = static_cast<R*>(out);
    if (nc == 4 && L >= 4) {  // the four components of a row pair in one CTA
      const int NP = L / 4;
      dim3 grd((nrows / 2 + NP - 1) / NP, 1);
      with_lines(L, [&](auto lc) {
        constexpr int LL = decltype(lc)::value;
        if constexpr (LL >= 4)
          with_shape<R, LL>(mp.fft[0], [&](auto sh) {
            launch_chained(k_fft_x_c2r<R, LL, 4, decltype(sh)>, grd, decltype(sh)::template threads<LL>(), sm, st, B1,
                           o, n1, nrows, g.K1, nc, mp.fft[0]);
          });
      });
    } else {  // one component per CTA row (grid.y = component)
      dim3 grd((nrows / 2 + L - 1) / L, nc);
      with_lines(L, [&](auto lc) {
        constexpr int LL = decltype(lc)::value;
        with_shape<R, LL>(mp.fft[0], [&](auto sh) {
          launch_chained(k_fft_x_c2r<R, LL, 1, decltype(sh)>, grd, decltype(sh)::template threads<LL>(), sm, st, B1, o,
                         n1, nrows, g.K1, nc, mp.fft[0]);
        });
      });
    }
    ++g_launches;
  }
}

template <typename... K>
void allow_smem(K... kernels) {
  (cudaFuncSetAttribute(kernels, cudaFuncAttributeMaxDynamicSharedMemorySize,
                        static_cast<int>(kSmemBudget + 16 * 1024)),
   ...);
}

template <typename R, int L>
void allow_lines() {
  allow_smem(k_fft_x_r2c<R, L>, k_fft_y_fwd<R, L>, k_fft_z_influence<R, L, false>,
             k_fft_z_influence<R, L, true>, k_fft_y_inv<R, L>,
             k_fft_x_c2r<R, L, 1>);
  allow_smem(k_fft_x_r2c_seg<R, L>, k_fft_y_fwd_seg<R, L>, k_fft_z_influence_seg<R, L>,
             k_fft_y_inv_seg<R, L>, k_fft_x_c2r_seg<R, L, 1>);
}

template <typename R, int L, class SH>
void allow_shape() {
  allow_smem(k_fft_x_r2c<R, L, SH>, k_fft_y_fwd<R, L, SH>, k_fft_z_influence<R, L, false, SH>,
             k_fft_z_influence<R, L, true, SH>, k_fft_y_inv<R, L, SH>, k_fft_x_c2r<R, L, 1, SH>,
             k_fft_x_c2r<R, L, 4, SH>);
  allow_smem(k_fft_x_r2c_seg<R, L, SH>, k_fft_y_fwd_seg<R, L, SH>, k_fft_z_influence_seg<R, L, SH>,
             k_fft_y_inv_seg<R, L, SH>, k_fft_x_c2r_seg<R, L, 1, SH>, k_fft_x_c2r_seg<R, L, 4, SH>);
}

template <typename R>
void allow_all() {
  if constexpr (sizeof(R) == 8) {
    allow_shape<R, 4, StatShape<280, 7, 5, 8, 40>>();
    allow_shape<R, 4, StatShape<512, 8, 8, 8, 64>>();
    allow_shape<R, 8, StatShape<128, 8, 8, 2>>();
  } else {
    allow_shape<R, 8, StatShape<140, 7, 5, 4, 36>>();
    allow_shape<R, 8, StatShape<160, 5, 8, 4, 40>>();
    allow_shape<R, 8, StatShape<280, 7, 5, 8, 40>>();
  }
  allow_lines<R, 8>();
  allow_lines<R, 4>();
  allow_lines<R, 2>();
  allow_lines<R, 1>();
  allow_smem(k_fft_x_c2r<R, 8, 4>, k_fft_x_c2r<R, 4, 4>);
  allow_smem(k_fft_x_c2r_seg<R, 8, 4>, k_fft_x_c2r_seg<R, 4, 4>);
}

// Segmented passes of a batch: lines per CTA b.L for every cell, shared
// memory for the batch's largest length per axis.
// The shape of axis d for a segmented launch: the compile-time one when every
// cell has the same length along d (and it is specialised), else generic.
template <typename R, int L, typename F>
void with_seg_shape(const BatchLaunch& b, int d, F&& f) {
  if (b.uniform[d])
    with_shape<R, L>(b.plan[d], f);
  else
    f(DynShape{});
}

template <typename R>
void forward_seg_impl(const BatchLaunch& b, cudaStream_t st) {
  const int nz = b.nc == 4 ? 2 : 1;
  with_lines(b.L, [&](auto lc) {
    constexpr int LL = decltype(lc)::value;
    if (b.n_r2c)
      with_seg_shape<R, LL>(b, 0, [&](auto sh) {
        using SH = decltype(sh);
        launch_chained(k_fft_x_r2c_seg<R, LL, SH>, b.n_r2c, SH::template threads<LL>(), b.smem[0],
                       st, b.cells, b.p_r2c, b.ncells);
      });
    if (b.n_yfwd)
      with_seg_shape<R, LL>(b, 1, [&](auto sh) {
        using SH = decltype(sh);
        launch_chained(k_fft_y_fwd_seg<R, LL, SH>, b.n_yfwd, SH::template threads<LL>(), b.smem[1],
                       st, b.cells, b.p_yfwd, b.ncells);
      });
    if (b.n_z)
      with_seg_shape<R, LL>(b, 2, [&](auto sh) {
        using SH = decltype(sh);
        launch_chained(k_fft_z_influence_seg<R, LL, SH>, b.n_z, SH::template threads<LL>(),
                       b.smem_z, st, b.cells, b.p_z, b.ncells, nz);
      });
  });
  g_launches += 3;
}

template <typename R>
void inverse_seg_impl(const BatchLaunch& b, cudaStream_t st) {
  with_lines(b.L, [&](auto lc) {
    constexpr int LL = decltype(lc)::value;
    if (b.n_yinv)
      with_seg_shape<R, LL>(b, 1, [&](auto sh) {
        using SH = decltype(sh);
        launch_chained(k_fft_y_inv_seg<R, LL, SH>, b.n_yinv, SH::template threads<LL>(), b.smem[1],
                       st, b.cells, b.p_yinv, b.ncells);
      });
    if (b.n_c2r)
      with_seg_shape<R, LL>(b, 0, [&](auto sh) {
        using SH = decltype(sh);
        if constexpr (LL >= 4) {
          if (b.nc == 4) {
            launch_chained(k_fft_x_c2r_seg<R, LL, 4, SH>, b.n_c2r, SH::template threads<LL>(),
                           b.smem[0], st, b.cells, b.p_c2r, b.ncells, b.nc);
            return;
          }
        }
        launch_chained(k_fft_x_c2r_seg<R, LL, 1, SH>, b.n_c2r, SH::template threads<LL>(),
                       b.smem[0], st, b.cells, b.p_c2r, b.ncells, b.nc);
      });
  });
  g_launches += 2;
}

}  // namespace

void mesh_pass_blocks(const MeshGeom& g, int L, int nc, int out[5]) { pass_blocks(g, L, nc, out); }

int mesh_batch_lines(int n, bool mixed, int extra) {
  return pick_lines(n, mixed ? sizeof(cx<float>) : sizeof(cx<double>), extra);
}

size_t mesh_pass_smem(int n, int L, bool mixed, int extra) {
  return pass_smem(n, L, mixed ? sizeof(cx<float>) : sizeof(cx<double>), extra);
}

void launch_forward_and_weight_seg(const BatchLaunch& b, cudaStream_t st) {
  if (b.mixed)
    forward_seg_impl<float>(b, st);
  else
    forward_seg_impl<double>(b, st);
}

void launch_inverse_seg(const BatchLaunch& b, cudaStream_t st) {
  if (b.mixed)
    inverse_seg_impl<float>(b, st);
  else
    inverse_seg_impl<double>(b, st);
}

int mesh_check_lengths(const MeshGeom& g, bool mixed) {
  const size_t cb = mixed ? sizeof(cx<float>) : sizeof(cx<double>);
  if (pick_lines(g.n[0], cb) == 0 || pick_lines(g.n[1], cb) == 0 ||
      pick_lines(g.n[2], cb, g.K3) == 0)
    return EWG_ERR_GRID_TOO_LARGE;
  return EWG_OK;
}

int mesh_configure_kernels() {
  allow_all<double>();
  allow_all<float>();
  return cudaGetLastError() == cudaSuccess ? EWG_OK : EWG_ERR_CUDA;
}

void launch_forward_and_weight(const MeshPlan& mp, const void* grid, void* A1, void* A2, void* B2,
                               int nc, cudaStream_t st, double* stress_part) {
  if (mp.mixed)
    forward_impl<float>(mp, grid, A1, A2, B2, nc, stress_part, st);
  else
    forward_impl<double>(mp, grid, A1, A2, B2, nc, stress_part, st);
}

void launch_inverse(const MeshPlan& mp, const void* B2, void* B1, void* out, int nc,
                    cudaStream_t st) {
  if (mp.mixed)
    inverse_impl<float>(mp, B2, B1, out, nc, st);
  else
    inverse_impl<double>(mp, B2, B1, out, nc, st);
}

void prof_mark(Profiler* p, cudaStream_t st, int stage) {
  if (!p || !p->on) return;
  if (p->n >= Profiler::kMax) return;
  if (!p->ev[p->n]) cudaEventCreate(&p->ev[p->n]);
  cudaEventRecord(p->ev[p->n], st);
  p->tag[p->n] = stage;
  p->launch_mark[p->n] = g_launches;
  ++p->n;
}

void prof_collect(Profiler* p) {
  if (!p || !p->on) return;
  for (int i = 0; i + 1 < p->n; ++i) {
    if (p->tag[i] < 0) continue;
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, p->ev[i], p->ev[i + 1]) == cudaSuccess) p->ms[p->tag[i]] += ms;
    p->launches[p->tag[i]] += p->launch_mark[i + 1] - p->launch_mark[i];
  }
  cudaGetLastError();
  p->n = 0;
}

MeshSizes mesh_sizes(const MeshGeom& g, const StencilDims& sd, int mixed, int nc, int natoms,
                     int nparts) {
  const size_t r = mixed ? 4 : 8, c = 2 * r;
  const size_t n1 = g.n[0], n2 = g.n[1], n3 = g.n[2];
  MeshSizes s;
  s.grid = n1 * n2 * n3 * r;
  s.A1 = n3 * n2 * g.K1 * c;
  s.A2 = n3 * g.K2 * g.K1 * c;
  const size_t nz = nc == 4 ? 2 : 1, ny = nc == 4 ? 3 : 1;  // force grids in the fractional basis
  s.B2 = nz * n3 * g.K2 * g.K1 * c;
  s.B1 = ny * n3 * n2 * g.K1 * c;
  s.out = nc * n1 * n2 * n3 * r;
  s.wtab = static_cast<size_t>(natoms) * sd.wstride * r;
  s.qk = static_cast<size_t>(natoms) * r;
  s.slot = static_cast<size_t>(natoms) * 16;
  s.part = static_cast<size_t>(natoms) * sd.S[0] * sd.S[1] * sd.S[2] * nparts * 8;
  return s;
}

}  // namespace ewg
