// ewg_fft.cuh -- shared-memory Stockham FFT for the mesh transforms.
//
// A CTA transforms L complex lines of length n, ping-ponging between two
// shared buffers.  Each pass of radix r and current sub-length p (Stockham
// autosort, decimation in time) reads the r inputs spaced n/r apart,
// multiplies input j by w^(j k) with w = exp(sign 2 pi i/(p r)) and k = i mod p,
// does an r-point DFT and writes output j to (i - k) r + k + j p.  After the
// last pass the data are in natural order.  Twiddles come from one table
// tw[e] = exp(-2 pi i e / n) per length; the inverse direction conjugates them.
// Radices 2, 3, 4, 5, 7, 8 are specialised; other odd primes up to 31 use a
// generic pass.  No normalisation is applied, matching the reference's FFTW
// usage (nfft/fft_backend.f90:43-58).
#pragma once

#include <cuda_runtime.h>

#include "ewg_internal.h"

namespace ewg {

template <typename R>
struct __align__(2 * sizeof(R)) cx {
  R x, y;
};

template <typename R>
__device__ __forceinline__ cx<R> mk(R x, R y) {
  cx<R> c;
  c.x = x;
  c.y = y;
  return c;
}
template <typename R>
__device__ __forceinline__ cx<R> add(cx<R> a, cx<R> b) {
  return mk(a.x + b.x, a.y + b.y);
}
template <typename R>
__device__ __forceinline__ cx<R> sub(cx<R> a, cx<R> b) {
  return mk(a.x - b.x, a.y - b.y);
}
template <typename R>
__device__ __forceinline__ cx<R> mul(cx<R> a, cx<R> b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// multiply by SIGN * i
template <typename R, int SIGN>
__device__ __forceinline__ cx<R> mul_si(cx<R> a) {
  return SIGN > 0 ? mk(-a.y, a.x) : mk(a.y, -a.x);
}
template <typename R>
__device__ __forceinline__ cx<R> scale(cx<R> a, R s) {
  return mk(a.x * s, a.y * s);
}

template <typename R>
__device__ __forceinline__ cx<R> twiddle(const cx<R>* __restrict__ tw, int e, int sign) {
  cx<R> w = tw[e];
  if (sign > 0) w.y = -w.y;
  return w;
}

// ---- small DFT kernels -----------------------------------------------------
template <typename R, int SIGN>
__device__ __forceinline__ void dft2(cx<R>* u) {
  cx<R> a = u[0], b = u[1];
  u[0] = add(a, b);
  u[1] = sub(a, b);
}

template <typename R, int SIGN>
__device__ __forceinline__ void dft4(cx<R>& a0, cx<R>& a1, cx<R>& a2, cx<R>& a3) {
  cx<R> s02 = add(a0, a2), d02 = sub(a0, a2);
  cx<R> s13 = add(a1, a3), d13 = mul_si<R, SIGN>(sub(a1, a3));
  a0 = add(s02, s13);
  a2 = sub(s02, s13);
  a1 = add(d02, d13);
  a3 = sub(d02, d13);
}

template <typename R, int SIGN>
__device__ __forceinline__ void dft3(cx<R>* u) {
  const R half = R(0.5);
  const R s3 = R(0.86602540378443864676);  // sqrt(3)/2
  cx<R> t1 = add(u[1], u[2]);
  cx<R> t2 = scale(mul_si<R, SIGN>(sub(u[1], u[2])), s3);
  cx<R> base = sub(u[0], scale(t1, half));
  u[0] = add(u[0], t1);
  u[1] = add(base, t2);
  u[2] = sub(base, t2);
}

template <typename R, int SIGN>
__device__ __forceinline__ void dft8(cx<R>* u) {
  const R r2 = R(0.70710678118654752440);  // 1/sqrt(2)
  cx<R> e0 = u[0], e1 = u[2], e2 = u[4], e3 = u[6];
  cx<R> o0 = u[1], o1 = u[3], o2 = u[5], o3 = u[7];
  dft4<R, SIGN>(e0, e1, e2, e3);
  dft4<R, SIGN>(o0, o1, o2, o3);
  // w = exp(SIGN 2 pi i / 8)
  cx<R> w1o = scale(add(o1, mul_si<R, SIGN>(o1)), r2);            // (1 + s i)/sqrt2
  cx<R> w2o = mul_si<R, SIGN>(o2);                                 // s i
  cx<R> w3o = scale(sub(mul_si<R, SIGN>(o3), o3), r2);            // (-1 + s i)/sqrt2
  u[0] = add(e0, o0);
  u[4] = sub(e0, o0);
  u[1] = add(e1, w1o);
  u[5] = sub(e1, w1o);
  u[2] = add(e2, w2o);
  u[6] = sub(e2, w2o);
  u[3] = add(e3, w3o);
  u[7] = sub(e3, w3o);
}

// Odd radix RR via conjugate-symmetric pairs; cos/sin of 2 pi j / RR are
// constants for RR = 5, 7 and read from the length-n twiddle table
// (tw[j n / RR] = exp(-2 pi i j / RR)) otherwise.
// cos and sin of 2 pi j / RR for the specialised odd radices (j = 1 .. (RR-1)/2).
__host__ __device__ constexpr double odd_root_cos(int rr, int j) {
  return rr == 5 ? (j == 1 ? 0.30901699437494742408 : -0.80901699437494742410)
                 : (j == 1 ? 0.62348980185873353053
                           : (j == 2 ? -0.22252093395631440429 : -0.90096886790241912624));
}
__host__ __device__ constexpr double odd_root_sin(int rr, int j) {
  return rr == 5 ? (j == 1 ? 0.95105651629515357212 : 0.58778525229247312917)
                 : (j == 1 ? 0.78183148246802980871
                           : (j == 2 ? 0.97492791218182360702 : 0.43388373911755812048));
}

template <typename R, int SIGN, int RR>
__device__ __forceinline__ void dft_odd(cx<R>* u, const cx<R>* __restrict__ tw, int n) {
  constexpr int H = (RR - 1) / 2;
  R c[H + 1], s[H + 1];
#pragma unroll
  for (int j = 1; j <= H; ++j) {
    if constexpr (RR == 5 || RR == 7) {
      c[j] = static_cast<R>(odd_root_cos(RR, j));
      s[j] = static_cast<R>(odd_root_sin(RR, j));
    } else {
      cx<R> w = tw[j * (n / RR)];
      c[j] = w.x;
      s[j] = -w.y;
    }
  }
  cx<R> sp[H + 1], sm[H + 1];
  cx<R> total = u[0];
#pragma unroll
  for (int j = 1; j <= H; ++j) {
    sp[j] = add(u[j], u[RR - j]);
    sm[j] = sub(u[j], u[RR - j]);
    total = add(total, sp[j]);
  }
  cx<R> out[RR];
  out[0] = total;
#pragma unroll
  for (int k = 1; k < RR; ++k) {
    cx<R> acc = u[0];
#pragma unroll
    for (int j = 1; j <= H; ++j) {
      const int idx = (j * k) % RR;
      const R cs = idx <= H ? c[idx] : c[RR - idx];
      const R sn = idx <= H ? s[idx] : -s[RR - idx];
      acc.x += sp[j].x * cs - R(SIGN) * sm[j].y * sn;
      acc.y += sp[j].y * cs + R(SIGN) * sm[j].x * sn;
    }
    out[k] = acc;
  }
#pragma unroll
  for (int k = 0; k < RR; ++k) u[k] = out[k];
}

template <typename R, int SIGN, int RR>
__device__ __forceinline__ void dft_fixed(cx<R>* u, const cx<R>* __restrict__ tw, int n) {
  if constexpr (RR == 2) {
    dft2<R, SIGN>(u);
  } else if constexpr (RR == 3) {
    dft3<R, SIGN>(u);
  } else if constexpr (RR == 4) {
    dft4<R, SIGN>(u[0], u[1], u[2], u[3]);
  } else if constexpr (RR == 8) {
    dft8<R, SIGN>(u);
  } else {
    dft_odd<R, SIGN, RR>(u, tw, n);
  }
}

template <typename R>
__device__ __forceinline__ const cx<R>* plan_twiddles(const FftPlan& plan);
template <>
__device__ __forceinline__ const cx<double>* plan_twiddles<double>(const FftPlan& plan) {
  return reinterpret_cast<const cx<double>*>(plan.tw64);
}
template <>
__device__ __forceinline__ const cx<float>* plan_twiddles<float>(const FftPlan& plan) {
  return reinterpret_cast<const cx<float>*>(plan.tw32);
}

}  // namespace ewg

namespace ewg {

// ---------------------------------------------------------------------------
// Line-fastest transforms with register edges.  A CTA transforms L lines (L a
// power of two) of length n; element e of line l sits at buf[e * L + l], the
// order in which the strided mesh axes find their lines in memory (consecutive
// k1), so global accesses are coalesced across the lines.  Threads map to
// (line, butterfly) with the line fastest.
//
// The first pass takes its inputs straight from a load functor (global memory
// or another shared buffer) and the last pass hands its outputs to a store
// functor, so only the passes in between go through the two ping-pong
// buffers.  With radices ordered odd first (the host factorisation does so),
// every shared-memory access of a pass is conflict-free for L = 8 and L = 4.
//
//   load(line, e)                 -> cx<R>   input element e of line `line`
//   store(line, e, v, spare)                 output element e; `spare` is a
//                                            shared buffer of n * L elements
//                                            that the transform no longer uses
//
// The caller synchronises before the call if the buffers (or data the load
// functor reads from shared memory) were written by other threads; the
// function ends without a barrier after the last pass.
// ---------------------------------------------------------------------------
template <typename R, int SIGN, int RR, int L, class Load, class Store>
__device__ __forceinline__ void edge_pass(const cx<R>* __restrict__ in, cx<R>* __restrict__ out,
                                          cx<R>* spare, int n, int p, bool first, bool last,
                                          const cx<R>* __restrict__ tw, Load& load, Store& store) {
  const int nr = n / RR;
  const int step = n / (p * RR);
  const int line = threadIdx.x & (L - 1);
  const int istep = blockDim.x / L;
  int i = threadIdx.x / L;
  int j = i / p, k = i - j * p;
  const int dj = istep / p, dk = istep - dj * p;
  for (; i < nr; i += istep) {
    cx<R> u[RR];
    if (first) {
#pragma unroll
      for (int jj = 0; jj < RR; ++jj) u[jj] = load(line, i + jj * nr);
    } else {
      const cx<R>* src = in + i * L + line;
#pragma unroll
      for (int jj = 0; jj < RR; ++jj) u[jj] = src[jj * nr * L];
      if (p > 1) {
        if constexpr (sizeof(R) == 8) {
          // FP64: one table read, the other powers by recurrence (error a few ulp).
          const cx<R> w1 = twiddle(tw, k * step, SIGN);
          cx<R> w = w1;
#pragma unroll
          for (int jj = 1; jj < RR; ++jj) {
            u[jj] = mul(u[jj], w);
            if (jj + 1 < RR) w = mul(w, w1);
          }
        } else {
#pragma unroll
          for (int jj = 1; jj < RR; ++jj) u[jj] = mul(u[jj], twiddle(tw, jj * k * step, SIGN));
        }
      }
    }
    dft_fixed<R, SIGN, RR>(u, tw, n);
    const int e0 = j * p * RR + k;
    if (last) {
#pragma unroll
      for (int jj = 0; jj < RR; ++jj) store(line, e0 + jj * p, u[jj], spare);
    } else {
      cx<R>* dst = out + e0 * L + line;
#pragma unroll
      for (int jj = 0; jj < RR; ++jj) dst[jj * p * L] = u[jj];
    }
    k += dk;
    j += dj;
    if (k >= p) {
      k -= p;
      ++j;
    }
  }
}

// Generic odd prime radix rr (slow path for lengths that only the reference's
// overrides can produce).
template <typename R, int SIGN, int L, class Load, class Store>
__device__ void edge_pass_generic(const cx<R>* __restrict__ in, cx<R>* __restrict__ out,
                                  cx<R>* spare, int n, int p, int rr, bool first, bool last,
                                  const cx<R>* __restrict__ tw, Load& load, Store& store) {
  const int nr = n / rr;
  const int step = n / (p * rr);
  const int line = threadIdx.x & (L - 1);
  for (int i = threadIdx.x / L; i < nr; i += blockDim.x / L) {
    const int k = i % p, j = i / p;
    const int e0 = j * p * rr + k;
    for (int s = 0; s < rr; ++s) {
      cx<R> acc = mk(R(0), R(0));
      for (int jj = 0; jj < rr; ++jj) {
        cx<R> v = first ? load(line, i + jj * nr) : in[(i + jj * nr) * L + line];
        if (!first && p > 1 && jj > 0) v = mul(v, twiddle(tw, jj * k * step, SIGN));
        acc = add(acc, mul(v, twiddle(tw, ((jj * s) % rr) * nr, SIGN)));
      }
      if (last)
        store(line, e0 + s * p, acc, spare);
      else
        out[(e0 + s * p) * L + line] = acc;
    }
  }
}

// ---------------------------------------------------------------------------
// The same passes with the length, the radix schedule, the sub-length p and
// the CTA size known at compile time: every index, loop bound and twiddle
// offset folds to a constant and the butterfly loops unroll.  Arithmetic and
// order are those of edge_pass, so results are bitwise the same.
// ---------------------------------------------------------------------------
template <typename R, int SIGN, int RR, int L, int T, int N, int P, bool FIRST, bool LAST,
          class Load, class Store>
__device__ __forceinline__ void edge_pass_s(const cx<R>* __restrict__ in, cx<R>* __restrict__ out,
                                            cx<R>* spare, const cx<R>* __restrict__ tw,
                                            Load& load, Store& store) {
  constexpr int NR = N / RR;
  constexpr int STEP = N / (P * RR);
  constexpr int ISTEP = T / L;
  constexpr int ITERS = (NR + ISTEP - 1) / ISTEP;
  const int line = threadIdx.x & (L - 1);
  const int i0 = threadIdx.x / L;
#pragma unroll
  for (int it = 0; it < ITERS; ++it) {
    const int i = i0 + it * ISTEP;
    if (NR % ISTEP != 0 && i >= NR) break;
    const int j = i / P, k = i - j * P;
    cx<R> u[RR];
    if (FIRST) {
#pragma unroll
      for (int jj = 0; jj < RR; ++jj) u[jj] = load(line, i + jj * NR);
    } else {
      const cx<R>* src = in + i * L + line;
#pragma unroll
      for (int jj = 0; jj < RR; ++jj) u[jj] = src[jj * NR * L];
      if (P > 1) {
        if constexpr (sizeof(R) == 8) {
          const cx<R> w1 = twiddle(tw, k * STEP, SIGN);
          cx<R> w = w1;
#pragma unroll
          for (int jj = 1; jj < RR; ++jj) {
            u[jj] = mul(u[jj], w);
            if (jj + 1 < RR) w = mul(w, w1);
          }
        } else {
#pragma unroll
          for (int jj = 1; jj < RR; ++jj) u[jj] = mul(u[jj], twiddle(tw, jj * k * STEP, SIGN));
        }
      }
    }
    dft_fixed<R, SIGN, RR>(u, tw, N);
    const int e0 = j * P * RR + k;
    if (LAST) {
#pragma unroll
      for (int jj = 0; jj < RR; ++jj) store(line, e0 + jj * P, u[jj], spare);
    } else {
      cx<R>* dst = out + e0 * L + line;
#pragma unroll
      for (int jj = 0; jj < RR; ++jj) dst[jj * P * L] = u[jj];
    }
  }
}

// Three passes of radices R0, R1, R2 (N = R0 R1 R2, in the host factorisation's
// order) on T threads; buffers as in fft_edges: the last pass's spare is a.
template <typename R, int SIGN, int L, int T, int N, int R0, int R1, int R2, class Load,
          class Store>
__device__ __forceinline__ void fft_static3(cx<R>* a, cx<R>* b, const cx<R>* __restrict__ tw,
                                            Load load, Store store) {
  static_assert(R0 * R1 * R2 == N, "radix schedule");
  edge_pass_s<R, SIGN, R0, L, T, N, 1, true, false>(b, a, a, tw, load, store);
  __syncthreads();
  edge_pass_s<R, SIGN, R1, L, T, N, R0, false, false>(a, b, b, tw, load, store);
  __syncthreads();
  edge_pass_s<R, SIGN, R2, L, T, N, R0 * R1, false, true>(b, a, a, tw, load, store);
}

template <typename R, int SIGN, int L, class Load, class Store>
__device__ void fft_edges(cx<R>* a, cx<R>* b, int n, const FftPlan& plan,
                          const cx<R>* __restrict__ tw, Load load, Store store) {
  int p = 1;
  cx<R>* src = b;  // unused by the first pass
  cx<R>* dst = a;
  const int ns = plan.nstages;
  for (int s = 0; s < ns; ++s) {
    const int rr = plan.radix[s];
    const bool first = s == 0, last = s == ns - 1;
    // Before the last pass, `dst` is the buffer its outputs would have used.
    cx<R>* spare = dst;
    switch (rr) {
      case 2: edge_pass<R, SIGN, 2, L>(src, dst, spare, n, p, first, last, tw, load, store); break;
      case 3: edge_pass<R, SIGN, 3, L>(src, dst, spare, n, p, first, last, tw, load, store); break;
      case 4: edge_pass<R, SIGN, 4, L>(src, dst, spare, n, p, first, last, tw, load, store); break;
      case 5: edge_pass<R, SIGN, 5, L>(src, dst, spare, n, p, first, last, tw, load, store); break;
      case 7: edge_pass<R, SIGN, 7, L>(src, dst, spare, n, p, first, last, tw, load, store); break;
      case 8: edge_pass<R, SIGN, 8, L>(src, dst, spare, n, p, first, last, tw, load, store); break;
      default:
        edge_pass_generic<R, SIGN, L>(src, dst, spare, n, p, rr, first, last, tw, load, store);
        break;
    }
    if (!last) __syncthreads();
    p *= rr;
    src = dst;
    dst = dst == a ? b : a;
  }
}

}  // namespace ewg
