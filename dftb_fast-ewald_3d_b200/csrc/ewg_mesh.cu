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
// the reference's mode set [-M/2, M/2-1]^3 (nfft/nfft.f90:61-75).  The force
// components use -i k_c c(k) Q(k).  Only k1 >= 0 is stored (Hermitian half).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "ewg_fft.cuh"
#include "ewg_kernels.h"

namespace ewg {

namespace {

constexpr int kSpreadTile = 16;
constexpr int kSpreadBatch = 32;
constexpr int kFftThreads = 256;
constexpr size_t kSmemBudget = 200 * 1024;

__device__ __forceinline__ int pmod(int a, int n) {
  int r = a % n;
  return r < 0 ? r + n : r;
}

template <typename R>
__device__ __forceinline__ void accumulate(double& acc, R s, R w) {
  if constexpr (sizeof(R) == 8) {
    acc = fma(static_cast<double>(s), static_cast<double>(w), acc);
  } else {
    acc += static_cast<double>(s * w);
  }
}

// ---------------------------------------------------------------------------
// Window weights (nfft/nfft.f90:122-159), evaluated in FP64 and stored in R.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void k_weights(const double4* __restrict__ fr, int n, int m, int W, double b,
                          double pref, R* __restrict__ wtab, R* __restrict__ qk) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double4 f = fr[k];
  const double fx[3] = {f.x, f.y, f.z};
  R* out = wtab + static_cast<size_t>(k) * 3 * W;
  for (int d = 0; d < 3; ++d)
    for (int o = -m; o <= m; ++o) {
      const double dd = fx[d] - static_cast<double>(o);
      out[d * W + o + m] = static_cast<R>(pref * exp(-(dd * dd) / b));
    }
  qk[k] = static_cast<R>(f.w);
}

// ---------------------------------------------------------------------------
// Spread.  A CTA owns a 16^3 tile of the fine grid; thread (py, pz) owns the
// x-pencil of 16 points at (y0+py, z0+pz) and keeps it in registers.  The atoms
// that can reach the tile live in a fixed set of home tiles (atoms are bucketed
// by the tile of their lowest stencil point); batches of them are staged in
// shared memory as per-tile folded weight vectors and applied as rank-1
// updates.  Every grid point is written once by its owner: no atomics, no
// zeroing pass, and a summation order fixed by the sorted atom order.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_spread(const int4* __restrict__ mc,
                                                const R* __restrict__ wtab,
                                                const R* __restrict__ qk,
                                                const int* __restrict__ tile_start, TileLists lx,
                                                TileLists ly, TileLists lz, int n1, int n2, int n3,
                                                int m, int W, R* __restrict__ grid) {
  constexpr int T = kSpreadTile;
  constexpr int B = kSpreadBatch;
  __shared__ R sW[3][B][T];
  __shared__ int sStart[64];
  __shared__ int sPrefix[65];
  __shared__ int sAtom[B];

  const int tx = blockIdx.x, ty = blockIdx.y, tz = blockIdx.z;
  const int org[3] = {tx * T, ty * T, tz * T};
  const int ext[3] = {min(T, n1 - org[0]), min(T, n2 - org[1]), min(T, n3 - org[2])};
  const int nn[3] = {n1, n2, n3};
  const int py = threadIdx.x % T, pz = threadIdx.x / T;

  double acc[T];
#pragma unroll
  for (int x = 0; x < T; ++x) acc[x] = 0.0;

  const int lenx = lx.len[tx], leny = ly.len[ty], lenz = lz.len[tz];
  const int nh = lenx * leny * lenz;
  for (int h0 = 0; h0 < nh; h0 += 64) {
    const int hc = min(64, nh - h0);
    __syncthreads();
    if (threadIdx.x < hc) {
      const int h = h0 + threadIdx.x;
      const int ix = h % lenx, iy = (h / lenx) % leny, iz = h / (lenx * leny);
      const int home = (lz.home[tz * lz.maxlen + iz] * ly.ntiles + ly.home[ty * ly.maxlen + iy]) *
                           lx.ntiles +
                       lx.home[tx * lx.maxlen + ix];
      const int s0 = tile_start[home];
      sStart[threadIdx.x] = s0;
      sPrefix[threadIdx.x + 1] = tile_start[home + 1] - s0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      sPrefix[0] = 0;
      for (int i = 1; i <= hc; ++i) sPrefix[i] += sPrefix[i - 1];
    }
    __syncthreads();
    const int total = sPrefix[hc];
    for (int b0 = 0; b0 < total; b0 += B) {
      const int nb = min(B, total - b0);
      if (threadIdx.x < nb) {
        const int f = b0 + threadIdx.x;
        int lo = 0, hi = hc - 1;  // last slot with prefix <= f
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (sPrefix[mid] <= f)
            lo = mid;
          else
            hi = mid - 1;
        }
        sAtom[threadIdx.x] = sStart[lo] + (f - sPrefix[lo]);
      }
      __syncthreads();
      for (int it = threadIdx.x; it < nb * 3 * T; it += blockDim.x) {
        const int a = it / (3 * T);
        const int r = it - a * 3 * T;
        const int d = r / T;
        const int p = r - d * T;
        const int k = sAtom[a];
        R w = R(0);
        if (p < ext[d]) {
          const int4 c4 = mc[k];
          const int c = d == 0 ? c4.x : (d == 1 ? c4.y : c4.z);
          int o = pmod(org[d] + p - c, nn[d]);
          while (o > m) o -= nn[d];
          const R* wk = wtab + (static_cast<size_t>(k) * 3 + d) * W;
          for (; o >= -m; o -= nn[d]) w += wk[o + m];
          if (d == 2) w *= qk[k];
        }
        sW[d][a][p] = w;
      }
      __syncthreads();
      for (int a = 0; a < nb; ++a) {
        const R s = sW[1][a][py] * sW[2][a][pz];
        if (s != R(0)) {
#pragma unroll
          for (int x = 0; x < T; ++x) accumulate<R>(acc[x], s, sW[0][a][x]);
        }
      }
      __syncthreads();
    }
  }
  if (py < ext[1] && pz < ext[2]) {
    R* row = grid + (static_cast<size_t>(org[2] + pz) * n2 + org[1] + py) * n1 + org[0];
#pragma unroll
    for (int x = 0; x < T; ++x)
      if (x < ext[0]) row[x] = static_cast<R>(acc[x]);
  }
}

// ---------------------------------------------------------------------------
// x pass, real to complex: two real rows per complex line; keep k1 = 0..K1-1.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(kFftThreads) k_fft_x_r2c(const R* __restrict__ grid,
                                                           cx<R>* __restrict__ A1, int n1,
                                                           int npairs, int K1, int P,
                                                           FftPlan plan) {
  extern __shared__ unsigned char smem_raw[];
  cx<R>* a = reinterpret_cast<cx<R>*>(smem_raw);
  cx<R>* b = a + static_cast<size_t>(P) * n1;
  const int pair0 = blockIdx.x * P;
  const int np = min(P, npairs - pair0);
  for (int t = threadIdx.x; t < np * n1; t += blockDim.x) {
    const int l = t / n1, k = t - l * n1;
    const size_t r0 = static_cast<size_t>(2 * (pair0 + l)) * n1;
    a[l * n1 + k] = mk(grid[r0 + k], grid[r0 + n1 + k]);
  }
  __syncthreads();
  const cx<R>* tw = plan_twiddles<R>(plan);
  cx<R>* res = fft_lines<R, -1>(a, b, n1, np, plan, tw);
  const R h = R(0.5);
  for (int t = threadIdx.x; t < np * K1; t += blockDim.x) {
    const int l = t / K1, k = t - l * K1;
    const cx<R> z = res[l * n1 + k];
    cx<R> zc = res[l * n1 + (k == 0 ? 0 : n1 - k)];
    zc.y = -zc.y;
    const size_t row = static_cast<size_t>(2 * (pair0 + l));
    A1[row * K1 + k] = mk(h * (z.x + zc.x), h * (z.y + zc.y));
    A1[(row + 1) * K1 + k] = mk(h * (z.y - zc.y), -h * (z.x - zc.x));
  }
}

// ---------------------------------------------------------------------------
// y pass, forward: lines over i2 for (i3, k1-block); keep k2 in [-M2/2, M2/2].
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(kFftThreads) k_fft_y_fwd(const cx<R>* __restrict__ A1,
                                                           cx<R>* __restrict__ A2, int n2, int K1,
                                                           int K2, int H2, int TK, FftPlan plan) {
  extern __shared__ unsigned char smem_raw[];
  cx<R>* a = reinterpret_cast<cx<R>*>(smem_raw);
  cx<R>* b = a + static_cast<size_t>(TK) * n2;
  const int k0 = blockIdx.x * TK;
  const int i3 = blockIdx.y;
  const int tk = min(TK, K1 - k0);
  for (int t = threadIdx.x; t < n2 * tk; t += blockDim.x) {
    const int i2 = t / tk, kk = t - i2 * tk;
    a[kk * n2 + i2] = A1[(static_cast<size_t>(i3) * n2 + i2) * K1 + k0 + kk];
  }
  __syncthreads();
  cx<R>* res = fft_lines<R, -1>(a, b, n2, tk, plan, plan_twiddles<R>(plan));
  const int h2 = H2;
  for (int t = threadIdx.x; t < K2 * tk; t += blockDim.x) {
    const int k2i = t / tk, kk = t - k2i * tk;
    const int idx = pmod(k2i - h2, n2);
    A2[(static_cast<size_t>(i3) * K2 + k2i) * K1 + k0 + kk] = res[kk * n2 + idx];
  }
}

// ---------------------------------------------------------------------------
// z pass forward, influence weights, z pass inverse -- fused per (k2, k1-block).
// ---------------------------------------------------------------------------
struct InfluenceArgs {
  int H[3];          // closed box |k_d| <= H_d
  int slo[3], shi[3];  // mode set S_d = [slo_d, shi_d] (nfft/nfft.f90:61-75)
  double rec[3][3];
  double prefactor;    // 4 pi / V
  double inv4a2;       // 1 / (4 alpha^2)
  const double* corr2[3];
};

template <typename R>
__global__ void __launch_bounds__(kFftThreads) k_fft_z_influence(
    const cx<R>* __restrict__ A2, cx<R>* __restrict__ B2, int n3, int K1, int K2, int K3, int TK,
    int nc, InfluenceArgs ia, FftPlan plan) {
  extern __shared__ unsigned char smem_raw[];
  cx<R>* a = reinterpret_cast<cx<R>*>(smem_raw);
  cx<R>* b = a + static_cast<size_t>(TK) * n3;
  cx<R>* q = b + static_cast<size_t>(TK) * n3;  // TK * K3 weighted modes
  const int k0 = blockIdx.x * TK;
  const int k2i = blockIdx.y;
  const int tk = min(TK, K1 - k0);
  const cx<R>* tw = plan_twiddles<R>(plan);
  for (int t = threadIdx.x; t < n3 * tk; t += blockDim.x) {
    const int i3 = t / tk, kk = t - i3 * tk;
    a[kk * n3 + i3] = A2[(static_cast<size_t>(i3) * K2 + k2i) * K1 + k0 + kk];
  }
  __syncthreads();
  cx<R>* res = fft_lines<R, -1>(a, b, n3, tk, plan, tw);
  const int h1 = ia.H[0], h2 = ia.H[1], h3 = ia.H[2];
  const int k2 = k2i - h2;
  const double twoPi = 2.0 * 3.14159265358979323846;
  for (int t = threadIdx.x; t < K3 * tk; t += blockDim.x) {
    const int k3i = t / tk, kk = t - k3i * tk;
    const int k1 = k0 + kk;
    const int k3 = k3i - h3;
    double wt = 0.0;
    if (!(k1 == 0 && k2 == 0 && k3 == 0)) {
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
      }
    }
    const cx<R> g = res[kk * n3 + pmod(k3, n3)];
    q[kk * K3 + k3i] = mk(static_cast<R>(wt * static_cast<double>(g.x)),
                          static_cast<R>(wt * static_cast<double>(g.y)));
  }
  __syncthreads();
  for (int c = 0; c < nc; ++c) {
    for (int t = threadIdx.x; t < n3 * tk; t += blockDim.x) {
      const int kk = t / n3, i3 = t - kk * n3;
      int k3;
      bool inside = true;
      if (i3 <= h3)
        k3 = i3;
      else if (i3 >= n3 - h3)
        k3 = i3 - n3;
      else {
        k3 = 0;
        inside = false;
      }
      cx<R> v = mk(R(0), R(0));
      if (inside) {
        v = q[kk * K3 + k3 + h3];
        if (c > 0) {
          const int k1 = k0 + kk;
          const R kc = static_cast<R>(twoPi * (k1 * ia.rec[0][c - 1] + k2 * ia.rec[1][c - 1] +
                                               k3 * ia.rec[2][c - 1]));
          v = mk(kc * v.y, -kc * v.x);  // -i kc v
        }
      }
      a[kk * n3 + i3] = v;
    }
    __syncthreads();
    cx<R>* r2 = fft_lines<R, 1>(a, b, n3, tk, plan, tw);
    cx<R>* dst = B2 + static_cast<size_t>(c) * n3 * K2 * K1;
    for (int t = threadIdx.x; t < n3 * tk; t += blockDim.x) {
      const int i3 = t / tk, kk = t - i3 * tk;
      dst[(static_cast<size_t>(i3) * K2 + k2i) * K1 + k0 + kk] = r2[kk * n3 + i3];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// y pass inverse: zero-padded k2 box -> i2, for (k1-block, i3, component).
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(kFftThreads) k_fft_y_inv(const cx<R>* __restrict__ B2,
                                                           cx<R>* __restrict__ B1, int n2, int n3,
                                                           int K1, int K2, int H2, int TK,
                                                           FftPlan plan) {
  extern __shared__ unsigned char smem_raw[];
  cx<R>* a = reinterpret_cast<cx<R>*>(smem_raw);
  cx<R>* b = a + static_cast<size_t>(TK) * n2;
  const int k0 = blockIdx.x * TK;
  const int i3 = blockIdx.y;
  const int c = blockIdx.z;
  const int tk = min(TK, K1 - k0);
  const int h2 = H2;
  const cx<R>* src = B2 + static_cast<size_t>(c) * n3 * K2 * K1;
  for (int t = threadIdx.x; t < n2 * tk; t += blockDim.x) {
    const int i2 = t / tk, kk = t - i2 * tk;
    int k2 = 0;
    bool inside = true;
    if (i2 <= h2)
      k2 = i2;
    else if (i2 >= n2 - h2)
      k2 = i2 - n2;
    else
      inside = false;
    a[kk * n2 + i2] =
        inside ? src[(static_cast<size_t>(i3) * K2 + k2 + h2) * K1 + k0 + kk] : mk(R(0), R(0));
  }
  __syncthreads();
  cx<R>* res = fft_lines<R, 1>(a, b, n2, tk, plan, plan_twiddles<R>(plan));
  cx<R>* dst = B1 + static_cast<size_t>(c) * n3 * n2 * K1;
  for (int t = threadIdx.x; t < n2 * tk; t += blockDim.x) {
    const int i2 = t / tk, kk = t - i2 * tk;
    dst[(static_cast<size_t>(i3) * n2 + i2) * K1 + k0 + kk] = res[kk * n2 + i2];
  }
}

// ---------------------------------------------------------------------------
// x pass, complex to real, all components of P row pairs; interleaved output.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(kFftThreads) k_fft_x_c2r(const cx<R>* __restrict__ B1,
                                                           R* __restrict__ out, int n1, int nrows,
                                                           int K1, int nc, int ncg, int P,
                                                           FftPlan plan) {
  // This CTA handles components [c0, c0 + ncg) of P row pairs.
  extern __shared__ unsigned char smem_raw[];
  const int pair0 = blockIdx.x * P;
  const int c0 = blockIdx.y * ncg;
  const int np = min(P, nrows / 2 - pair0);
  const int nl = np * ncg;  // line index = cc * np + l
  cx<R>* a = reinterpret_cast<cx<R>*>(smem_raw);
  cx<R>* b = a + static_cast<size_t>(P) * ncg * n1;
  for (int t = threadIdx.x; t < nl * n1; t += blockDim.x) {
    const int line = t / n1, k = t - line * n1;
    const int cc = line / np, l = line - cc * np;
    const size_t ra = static_cast<size_t>(2 * (pair0 + l));
    const cx<R>* src = B1 + static_cast<size_t>(c0 + cc) * nrows * K1;
    cx<R> fa = mk(R(0), R(0)), fb = mk(R(0), R(0));
    if (k < K1) {
      fa = src[ra * K1 + k];
      fb = src[(ra + 1) * K1 + k];
      if (k == 0) {
        fa.y = R(0);
        fb.y = R(0);
      }
    } else if (k > n1 - K1) {
      fa = src[ra * K1 + (n1 - k)];
      fb = src[(ra + 1) * K1 + (n1 - k)];
      fa.y = -fa.y;
      fb.y = -fb.y;
    }
    a[line * n1 + k] = mk(fa.x - fb.y, fa.y + fb.x);
  }
  __syncthreads();
  cx<R>* res = fft_lines<R, 1>(a, b, n1, nl, plan, plan_twiddles<R>(plan));
  for (int t = threadIdx.x; t < np * n1; t += blockDim.x) {
    const int l = t / n1, i1 = t - l * n1;
    const size_t ra = static_cast<size_t>(2 * (pair0 + l));
    R* oa = out + (ra * n1 + i1) * nc + c0;
    R* ob = out + ((ra + 1) * n1 + i1) * nc + c0;
    for (int cc = 0; cc < ncg; ++cc) {
      const cx<R> z = res[(cc * np + l) * n1 + i1];
      oa[cc] = z.x;
      ob[cc] = z.y;
    }
  }
}

// ---------------------------------------------------------------------------
// Gather: one warp per atom, lanes along o1, rows (o2, o3) in order.  Sum of
// w1 (w2 w3) g over the (2m+1)^3 stencil (nfft/nfft.f90:384-401), fused with
// the final assembly of potential and force.
// ---------------------------------------------------------------------------
template <typename R, int NC>
__global__ void __launch_bounds__(256) k_gather(const int4* __restrict__ mc,
                                                const R* __restrict__ wtab,
                                                const int* __restrict__ perm,
                                                const R* __restrict__ grid, int n1, int n2, int n3,
                                                int m, int W, int n, const double* __restrict__ q,
                                                double self_coef, const double* __restrict__ pot_sr,
                                                const double* __restrict__ f_sr,
                                                double* __restrict__ pot,
                                                double* __restrict__ force) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int4 c = mc[warp];
  const R* wt = wtab + static_cast<size_t>(warp) * 3 * W;
  double acc[NC];
#pragma unroll
  for (int j = 0; j < NC; ++j) acc[j] = 0.0;
  const int nlane = (W + 31) / 32;
  for (int o3 = 0; o3 < W; ++o3) {
    const int i3 = pmod(c.z + o3 - m, n3);
    const R w3 = wt[2 * W + o3];
    for (int o2 = 0; o2 < W; ++o2) {
      const int i2 = pmod(c.y + o2 - m, n2);
      const R s = wt[W + o2] * w3;
      const size_t rowbase = (static_cast<size_t>(i3) * n2 + i2) * n1;
      for (int li = 0; li < nlane; ++li) {
        const int o1 = lane + 32 * li;
        if (o1 < W) {
          const int i1 = pmod(c.x + o1 - m, n1);
          const R w = wt[o1] * s;
          const R* g = grid + (rowbase + i1) * NC;
#pragma unroll
          for (int j = 0; j < NC; ++j) accumulate<R>(acc[j], w, g[j]);
        }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < NC; ++j)
    for (int off = 16; off > 0; off >>= 1) acc[j] += __shfl_down_sync(0xffffffffu, acc[j], off);
  if (lane == 0) {
    const int i = perm[warp];
    const double qi = q[i];
    pot[i] = (pot_sr[i] + acc[0]) + self_coef * qi;
    if (NC == 4 && force) {
#pragma unroll
      for (int d = 0; d < 3; ++d) force[3 * i + d] = f_sr[3 * i + d] + qi * acc[1 + d];
    }
  }
}

template <typename R>
size_t cbytes() {
  return sizeof(cx<R>);
}

template <typename R>
void weights_impl(const MeshPlan& mp, const double4* fr, int n, void* wtab, void* qk,
                  cudaStream_t st) {
  if (n == 0) return;
  k_weights<R><<<(n + 127) / 128, 128, 0, st>>>(fr, n, mp.g.m, mp.g.W, mp.g.b, mp.g.pref,
                                                 static_cast<R*>(wtab), static_cast<R*>(qk));
  ++g_launches;
}

template <typename R>
void spread_impl(const MeshPlan& mp, const int4* mc, const void* wtab, const void* qk,
                 const int* tile_start, void* grid, cudaStream_t st) {
  dim3 grd(mp.ntiles[0], mp.ntiles[1], mp.ntiles[2]);
  k_spread<R><<<grd, 256, 0, st>>>(mc, static_cast<const R*>(wtab), static_cast<const R*>(qk),
                                    tile_start, mp.tl[0], mp.tl[1], mp.tl[2], mp.g.n[0],
                                    mp.g.n[1], mp.g.n[2], mp.g.m, mp.g.W, static_cast<R*>(grid));
  ++g_launches;
}

int lines_for(size_t per_line_bytes, int cap) {
  size_t l = kSmemBudget / std::max<size_t>(per_line_bytes, 1);
  return static_cast<int>(std::max<size_t>(1, std::min<size_t>(l, cap)));
}

template <typename R>
void forward_impl(const MeshPlan& mp, const void* grid, void* A1v, void* A2v, void* B2v, int nc,
                  cudaStream_t st) {
  const MeshGeom& g = mp.g;
  const int n1 = g.n[0], n2 = g.n[1], n3 = g.n[2];
  cx<R>* A1 = static_cast<cx<R>*>(A1v);
  cx<R>* A2 = static_cast<cx<R>*>(A2v);
  cx<R>* B2 = static_cast<cx<R>*>(B2v);
  const size_t cb = cbytes<R>();
  {  // x, real to complex
    prof_mark(mp.prof, st, ST_FFT_X_R2C);
    const int npairs = n2 * n3 / 2;
    const int P = lines_for(2 * n1 * cb, 8);
    const size_t sm = 2 * static_cast<size_t>(P) * n1 * cb;
    k_fft_x_r2c<R><<<(npairs + P - 1) / P, kFftThreads, sm, st>>>(static_cast<const R*>(grid), A1,
                                                                    n1, npairs, g.K1, P, mp.fft[0]);
    ++g_launches;
  }
  {  // y forward
    prof_mark(mp.prof, st, ST_FFT_Y_FWD);
    const int TK = lines_for(2 * n2 * cb, 8);
    const size_t sm = 2 * static_cast<size_t>(TK) * n2 * cb;
    dim3 grd((g.K1 + TK - 1) / TK, n3);
    k_fft_y_fwd<R><<<grd, kFftThreads, sm, st>>>(A1, A2, n2, g.K1, g.K2, (g.K2 - 1) / 2, TK,
                                                 mp.fft[1]);
    ++g_launches;
  }
  {  // z forward + influence + z inverse
    prof_mark(mp.prof, st, ST_FFT_Z_INFL);
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
    const int TK = lines_for((2 * n3 + g.K3) * cb, 8);
    const size_t sm = (2 * static_cast<size_t>(TK) * n3 + static_cast<size_t>(TK) * g.K3) * cb;
    dim3 grd((g.K1 + TK - 1) / TK, g.K2);
    k_fft_z_influence<R><<<grd, kFftThreads, sm, st>>>(A2, B2, n3, g.K1, g.K2, g.K3, TK, nc, ia,
                                                        mp.fft[2]);
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
    const int TK = lines_for(2 * n2 * cb, 8);
    const size_t sm = 2 * static_cast<size_t>(TK) * n2 * cb;
    dim3 grd((g.K1 + TK - 1) / TK, n3, nc);
    k_fft_y_inv<R><<<grd, kFftThreads, sm, st>>>(B2, B1, n2, n3, g.K1, g.K2, (g.K2 - 1) / 2, TK,
                                                 mp.fft[1]);
    ++g_launches;
  }
  {
    prof_mark(mp.prof, st, ST_FFT_X_C2R);
    const int nrows = n2 * n3;
    // All components of a row pair in one CTA when they fit, else one per CTA.
    const int ncg = 2 * static_cast<size_t>(nc) * n1 * cb <= kSmemBudget ? nc : 1;
    const int P = lines_for(2 * static_cast<size_t>(ncg) * n1 * cb, 4);
    const size_t sm = 2 * static_cast<size_t>(P) * ncg * n1 * cb;
    dim3 grd((nrows / 2 + P - 1) / P, nc / ncg);
    k_fft_x_c2r<R><<<grd, kFftThreads, sm, st>>>(B1, static_cast<R*>(out), n1, nrows, g.K1, nc, ncg,
                                                 P, mp.fft[0]);
    ++g_launches;
  }
}

template <typename R>
void gather_impl(const MeshPlan& mp, const int4* mc, const void* wtab, const int* perm,
                 const void* grid, int nc, int n, const double* q, double self_coef,
                 const double* pot_sr, const double* f_sr, double* pot, double* force,
                 cudaStream_t st) {
  if (n == 0) return;
  const int threads = 256;
  const int blocks = (n * 32 + threads - 1) / threads;
  const MeshGeom& g = mp.g;
  if (nc == 4)
    k_gather<R, 4><<<blocks, threads, 0, st>>>(mc, static_cast<const R*>(wtab), perm,
                                               static_cast<const R*>(grid), g.n[0], g.n[1], g.n[2],
                                               g.m, g.W, n, q, self_coef, pot_sr, f_sr, pot, force);
  else
    k_gather<R, 1><<<blocks, threads, 0, st>>>(mc, static_cast<const R*>(wtab), perm,
                                               static_cast<const R*>(grid), g.n[0], g.n[1], g.n[2],
                                               g.m, g.W, n, q, self_coef, pot_sr, f_sr, pot, nullptr);
  ++g_launches;
}

template <typename... K>
void allow_smem(K... kernels) {
  (cudaFuncSetAttribute(kernels, cudaFuncAttributeMaxDynamicSharedMemorySize,
                        static_cast<int>(kSmemBudget + 16 * 1024)),
   ...);
}

}  // namespace

int mesh_configure_kernels() {
  allow_smem(k_fft_x_r2c<double>, k_fft_y_fwd<double>, k_fft_z_influence<double>,
             k_fft_y_inv<double>, k_fft_x_c2r<double>, k_fft_x_r2c<float>, k_fft_y_fwd<float>,
             k_fft_z_influence<float>, k_fft_y_inv<float>, k_fft_x_c2r<float>);
  return cudaGetLastError() == cudaSuccess ? EWG_OK : EWG_ERR_CUDA;
}

void launch_weights(const MeshPlan& mp, const double4* fr, int n, void* wtab, void* qk,
                    cudaStream_t st) {
  if (mp.mixed)
    weights_impl<float>(mp, fr, n, wtab, qk, st);
  else
    weights_impl<double>(mp, fr, n, wtab, qk, st);
}

void launch_spread(const MeshPlan& mp, const int4* mc, const void* wtab, const void* qk,
                   const int* tile_start, void* grid, cudaStream_t st) {
  if (mp.mixed)
    spread_impl<float>(mp, mc, wtab, qk, tile_start, grid, st);
  else
    spread_impl<double>(mp, mc, wtab, qk, tile_start, grid, st);
}

void launch_forward_and_weight(const MeshPlan& mp, const void* grid, void* A1, void* A2, void* B2,
                               int nc, cudaStream_t st) {
  if (mp.mixed)
    forward_impl<float>(mp, grid, A1, A2, B2, nc, st);
  else
    forward_impl<double>(mp, grid, A1, A2, B2, nc, st);
}

void launch_inverse(const MeshPlan& mp, const void* B2, void* B1, void* out, int nc,
                    cudaStream_t st) {
  if (mp.mixed)
    inverse_impl<float>(mp, B2, B1, out, nc, st);
  else
    inverse_impl<double>(mp, B2, B1, out, nc, st);
}

void launch_gather(const MeshPlan& mp, const int4* mc, const void* wtab, const int* perm,
                   const void* grid, int nc, int n, const double* q, double self_coef,
                   const double* pot_sr, const double* f_sr, double* pot, double* force,
                   cudaStream_t st) {
  if (mp.mixed)
    gather_impl<float>(mp, mc, wtab, perm, grid, nc, n, q, self_coef, pot_sr, f_sr, pot, force, st);
  else
    gather_impl<double>(mp, mc, wtab, perm, grid, nc, n, q, self_coef, pot_sr, f_sr, pot, force,
                        st);
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

MeshSizes mesh_sizes(const MeshGeom& g, int mixed, int nc, int natoms) {
  const size_t r = mixed ? 4 : 8, c = 2 * r;
  const size_t n1 = g.n[0], n2 = g.n[1], n3 = g.n[2];
  MeshSizes s;
  s.grid = n1 * n2 * n3 * r;
  s.A1 = n3 * n2 * g.K1 * c;
  s.A2 = n3 * g.K2 * g.K1 * c;
  s.B2 = nc * n3 * g.K2 * g.K1 * c;
  s.B1 = nc * n3 * n2 * g.K1 * c;
  s.out = nc * n1 * n2 * n3 * r;
  s.wtab = static_cast<size_t>(natoms) * 3 * g.W * r;
  s.qk = static_cast<size_t>(natoms) * r;
  return s;
}

}  // namespace ewg
