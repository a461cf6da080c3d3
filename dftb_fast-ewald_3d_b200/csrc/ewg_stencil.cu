// ewg_stencil.cu -- the particle side of the NFFT: window weights, spread and
// gather (nfft/nfft.f90:122-159, :253-278, :380-402).
//
// Tiling.  The fine grid is cut into tiles of 8 x 16 x 16 points.  A CTA owns
// one tile; thread (py, pz) owns the x-pencil of 8 points at (y0+py, z0+pz)
// and keeps it in registers.  Atoms are bucketed by the tile that holds the
// lowest point of their stencil; the atoms that can reach a tile live in a
// fixed set of home tiles (per-axis lists, host-built).
//
// Weights.  Along each axis an atom's stencil [c-m, c+m] (mod n) touches a run
// of at most S_d consecutive tiles, starting at tile f_d.  The weights kernel
// stores, per atom and axis, the window weights already laid out per touched
// tile (S_d * T_d values, zero outside the stencil and beyond the grid end;
// points the stencil reaches twice on a small grid carry the sum).  A CTA then
// copies an atom's three weight vectors for its tile with no index arithmetic.
//
// Spread: each thread accumulates q w1 w2 w3 into its pencil, atom by atom in
// sorted order, and writes it once: no atomics, no zeroing, fixed order.
// Gather: each thread forms its pencil's contribution to a batch of atoms;
// a warp reduce-scatter sums the batch over the warp's pencils, the CTA sums its
// warps in order, and the per-(atom, tile) partial goes to its own slot; a final
// kernel adds each atom's slots in a fixed order.  Results are bitwise
// reproducible.

#include <cuda_runtime.h>

#include <type_traits>

#include "ewg_kernels.h"

namespace ewg {

namespace {

constexpr int TX = kTileX, TY = kTileY, TZ = kTileZ;
constexpr int kThreads = TY * TZ;  // one thread per x-pencil
static_assert(kThreads == 256, "tile shape assumes 256 threads");
constexpr int kWindow = 256;       // candidates tested per compaction window

__device__ __forceinline__ int pmod(int a, int n) {
  int r = a % n;
  return r < 0 ? r + n : r;
}

__device__ __forceinline__ int slot_first(int packed) { return packed & 0xffff; }
__device__ __forceinline__ int slot_count(int packed) { return packed >> 16; }

// ---------------------------------------------------------------------------
// Tiled window weights, one thread per (atom, axis).
// ---------------------------------------------------------------------------
template <typename R>
__global__ void k_weights_tiled(const int4* __restrict__ mc, const double4* __restrict__ fr, int n,
                                StencilDims sd, R* __restrict__ wtab, R* __restrict__ qk,
                                int4* __restrict__ slot) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 3 * n) return;
  const int k = idx / 3, d = idx - 3 * k;
  const int4 c4 = mc[k];
  const double4 f4 = fr[k];
  const int c = d == 0 ? c4.x : (d == 1 ? c4.y : c4.z);
  const double frac = d == 0 ? f4.x : (d == 1 ? f4.y : f4.z);
  const int nd = sd.n[d], T = sd.T[d], nt = sd.ntiles[d], S = sd.S[d];
  const int m = sd.m;
  // Tiles the stencil [c - m, c + m] (mod n) runs through, starting at `first`;
  // a stencil that comes back into its first tile, or covers the whole axis,
  // touches every tile once (repeated points are folded into the weights).
  int first, count;
  if (2 * m + 1 >= nd) {
    first = 0;
    count = nt;
  } else {
    const int p0 = pmod(c - m, nd);
    int t = p0 / T;
    first = t;
    int covered = min((t + 1) * T, nd) - p0;
    count = 1;
    while (covered < 2 * m + 1) {
      t = t + 1 == nt ? 0 : t + 1;
      ++count;
      covered += min((t + 1) * T, nd) - t * T;
    }
    count = min(count, nt);
  }
  R* out = wtab + static_cast<size_t>(k) * sd.wstride + sd.woff[d];
  for (int s = 0; s < S; ++s) {
    const int origin = ((first + s) % nt) * T;
    for (int p = 0; p < T; ++p) {
      const int P = origin + p;
      double w = 0.0;
      if (s < count && P < nd) {
        int o = pmod(P - c, nd);  // largest offset <= m congruent to P - c
        while (o > m) o -= nd;
        while (o + nd <= m) o += nd;
        for (; o >= -m; o -= nd) {
          const double dd = frac - static_cast<double>(o);
          w += sd.pref * exp(-(dd * dd) / sd.b);
        }
      }
      out[s * T + p] = static_cast<R>(w);
    }
  }
  int* sp = reinterpret_cast<int*>(&slot[k]);
  sp[d] = first | (count << 16);
  if (d == 0) {
    sp[3] = 0;
    qk[k] = static_cast<R>(f4.w);
  }
}

// ---------------------------------------------------------------------------
// Candidate enumeration shared by spread and gather: the atoms of the home
// tiles of this tile, filtered to those whose stencil reaches it, compacted in
// candidate order into sList (atom index) and sSlots (packed slot indices).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void load_home_chunk(const int* __restrict__ tile_start, const TileLists& lx,
                                                const TileLists& ly, const TileLists& lz, int tx,
                                                int ty, int tz, int h0, int hc, int* sStart,
                                                int* sPrefix) {
  const int lenx = lx.len[tx], leny = ly.len[ty];
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
}

// Tests candidates [w0, w0 + NT) of the chunk (NT = threads of the CTA);
// returns the number kept.
template <int NT = kThreads>
__device__ __forceinline__ int compact_window(const int4* __restrict__ slot, const StencilDims& sd,
                                              int tx, int ty, int tz, int w0, int total, int hc,
                                              const int* sStart, const int* sPrefix, int* sList,
                                              int* sSlots, int* sWarpCount) {
  const int f = w0 + threadIdx.x;
  int k = -1, packed = 0;
  bool keep = false;
  if (f < total) {
    int lo = 0, hi = hc - 1;  // last home slot with prefix <= f (non-empty by construction)
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (sPrefix[mid] <= f)
        lo = mid;
      else
        hi = mid - 1;
    }
    k = sStart[lo] + (f - sPrefix[lo]);
    const int4 si = slot[k];
    const int t3[3] = {tx, ty, tz};
    const int s3[3] = {si.x, si.y, si.z};
    keep = true;
    int sl[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      sl[d] = pmod(t3[d] - slot_first(s3[d]), sd.ntiles[d]);
      keep = keep && sl[d] < slot_count(s3[d]);
    }
    packed = sl[0] | (sl[1] << 8) | (sl[2] << 16);
  }
  const unsigned ballot = __ballot_sync(0xffffffffu, keep);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sWarpCount[wid] = __popc(ballot);
  __syncthreads();
  int base = 0, kept = 0;
  for (int w = 0; w < NT / 32; ++w) {
    const int cnt = sWarpCount[w];
    if (w < wid) base += cnt;
    kept += cnt;
  }
  if (keep) {
    const int pos = base + __popc(ballot & ((1u << lane) - 1u));
    sList[pos] = k;
    sSlots[pos] = packed;
  }
  __syncthreads();
  return kept;
}

// Copies batch atoms' per-tile weights into sW (layout [axis][a][T]).
template <typename R, int B>
__device__ __forceinline__ void fill_batch(const R* __restrict__ wtab, const R* __restrict__ qk,
                                           const StencilDims& sd, const int* sList,
                                           const int* sSlots, int b0, int nb, bool scale_q,
                                           R (*sW1)[TX], R (*sW2)[TY], R (*sW3)[TZ]) {
  constexpr int per = TX + TY + TZ;
  for (int it = threadIdx.x; it < nb * per; it += blockDim.x) {
    const int a = it / per;
    const int r = it - a * per;
    const int k = sList[b0 + a];
    const int ps = sSlots[b0 + a];
    const R* wk = wtab + static_cast<size_t>(k) * sd.wstride;
    if (r < TX) {
      sW1[a][r] = wk[sd.woff[0] + (ps & 0xff) * TX + r];
    } else if (r < TX + TY) {
      const int p = r - TX;
      sW2[a][p] = wk[sd.woff[1] + ((ps >> 8) & 0xff) * TY + p];
    } else {
      const int p = r - TX - TY;
      R w = wk[sd.woff[2] + ((ps >> 16) & 0xff) * TZ + p];
      if (scale_q) w *= qk[k];
      sW3[a][p] = w;
    }
  }
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
// Spread
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(kThreads) k_spread_tiles(
    const int4* __restrict__ slot, const R* __restrict__ wtab, const R* __restrict__ qk,
    const int* __restrict__ tile_start, TileLists lx, TileLists ly, TileLists lz, StencilDims sd,
    R* __restrict__ grid) {
  constexpr int B = 16;
  __shared__ R sW1[B][TX];
  __shared__ R sW2[B][TY];
  __shared__ R sW3[B][TZ];
  __shared__ int sStart[64];
  __shared__ int sPrefix[65];
  __shared__ int sList[kWindow];
  __shared__ int sSlots[kWindow];
  __shared__ int sWarpCount[kThreads / 32];

  const int tx = blockIdx.x, ty = blockIdx.y, tz = blockIdx.z;
  const int x0 = tx * TX, y0 = ty * TY, z0 = tz * TZ;
  const int py = threadIdx.x % TY, pz = threadIdx.x / TY;
  double acc[TX];
#pragma unroll
  for (int x = 0; x < TX; ++x) acc[x] = 0.0;

  const int nh = lx.len[tx] * ly.len[ty] * lz.len[tz];
  for (int h0 = 0; h0 < nh; h0 += 64) {
    const int hc = min(64, nh - h0);
    __syncthreads();
    load_home_chunk(tile_start, lx, ly, lz, tx, ty, tz, h0, hc, sStart, sPrefix);
    const int total = sPrefix[hc];
    for (int w0 = 0; w0 < total; w0 += kWindow) {
      const int kept = compact_window(slot, sd, tx, ty, tz, w0, total, hc, sStart, sPrefix, sList,
                                      sSlots, sWarpCount);
      for (int b0 = 0; b0 < kept; b0 += B) {
        const int nb = min(B, kept - b0);
        fill_batch<R, B>(wtab, qk, sd, sList, sSlots, b0, nb, true, sW1, sW2, sW3);
        __syncthreads();
        for (int a = 0; a < nb; ++a) {
          const R s = sW2[a][py] * sW3[a][pz];
          if (s != R(0)) {
#pragma unroll
            for (int x = 0; x < TX; ++x) accumulate<R>(acc[x], s, sW1[a][x]);
          }
        }
        __syncthreads();
      }
    }
  }
  const int ey = min(TY, sd.n[1] - y0), ez = min(TZ, sd.n[2] - z0), ex = min(TX, sd.n[0] - x0);
  if (py < ey && pz < ez) {
    R* row = grid + (static_cast<size_t>(z0 + pz) * sd.n[1] + y0 + py) * sd.n[0] + x0;
#pragma unroll
    for (int x = 0; x < TX; ++x)
      if (x < ex) row[x] = static_cast<R>(acc[x]);
  }
}

// ---------------------------------------------------------------------------
// Gather: per-(atom, tile) partial sums of w1 w2 w3 g over the tile for NC
// components, one thread per atom.  The tile's grid values sit in shared
// memory and every lane of a warp reads the same point at the same time (a
// broadcast), multiplying it by its own atom's weights; rows no lane of the
// warp reaches are skipped.  Each thread writes its atom's partial to the
// atom's slot for this tile, so no cross-thread reduction is needed.
// ---------------------------------------------------------------------------
constexpr int kGatherThreads = 128;

template <typename R, int NC>
__global__ void __launch_bounds__(kGatherThreads) k_gather_tiles(
    const int4* __restrict__ slot, const R* __restrict__ wtab, const int* __restrict__ tile_start,
    TileLists lx, TileLists ly, TileLists lz, StencilDims sd, const R* __restrict__ grid,
    double* __restrict__ part) {
  using V = typename std::conditional<NC == 4, typename std::conditional<sizeof(R) == 8, double4, float4>::type, R>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* sG = reinterpret_cast<V*>(smem_raw);  // [TZ][TY][TX]
  __shared__ int sStart[64];
  __shared__ int sPrefix[65];
  __shared__ int sList[kGatherThreads];
  __shared__ int sSlots[kGatherThreads];
  __shared__ int sWarpCount[kGatherThreads / 32];

  const int tx = blockIdx.x, ty = blockIdx.y, tz = blockIdx.z;
  const int x0 = tx * TX, y0 = ty * TY, z0 = tz * TZ;
  const int ex = min(TX, sd.n[0] - x0), ey = min(TY, sd.n[1] - y0), ez = min(TZ, sd.n[2] - z0);

  // Stage the tile (zero beyond the grid end).
  for (int t = threadIdx.x; t < TX * TY * TZ; t += blockDim.x) {
    const int x = t % TX, y = (t / TX) % TY, z = t / (TX * TY);
    V v;
    if (x < ex && y < ey && z < ez) {
      v = reinterpret_cast<const V*>(grid)[(static_cast<size_t>(z0 + z) * sd.n[1] + y0 + y) * sd.n[0] + x0 + x];
    } else {
      v = V();
      if constexpr (NC == 1) v = R(0);
    }
    sG[t] = v;
  }
  const int nslots = sd.S[0] * sd.S[1] * sd.S[2];
  const int nh = lx.len[tx] * ly.len[ty] * lz.len[tz];
  for (int h0 = 0; h0 < nh; h0 += 64) {
    const int hc = min(64, nh - h0);
    __syncthreads();
    load_home_chunk(tile_start, lx, ly, lz, tx, ty, tz, h0, hc, sStart, sPrefix);
    const int total = sPrefix[hc];
    for (int w0 = 0; w0 < total; w0 += kGatherThreads) {
      const int kept = compact_window<kGatherThreads>(slot, sd, tx, ty, tz, w0, total, hc, sStart,
                                                      sPrefix, sList, sSlots, sWarpCount);
      const bool active = threadIdx.x < kept;
      R w1[TX], w2[TY];
      int k = 0, ps = 0;
      const R* wk3 = nullptr;  // this atom's z weights for the tile (read through L1)
      if (active) {
        k = sList[threadIdx.x];
        ps = sSlots[threadIdx.x];
        const R* wk = wtab + static_cast<size_t>(k) * sd.wstride;
#pragma unroll
        for (int x = 0; x < TX; ++x) w1[x] = wk[sd.woff[0] + (ps & 0xff) * TX + x];
#pragma unroll
        for (int y = 0; y < TY; ++y) w2[y] = wk[sd.woff[1] + ((ps >> 8) & 0xff) * TY + y];
        wk3 = wk + sd.woff[2] + ((ps >> 16) & 0xff) * TZ;
      } else {
#pragma unroll
        for (int x = 0; x < TX; ++x) w1[x] = R(0);
#pragma unroll
        for (int y = 0; y < TY; ++y) w2[y] = R(0);
      }
      double acc[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[c] = 0.0;
      // Warps with no atom skip the whole tile (warp-uniform).
      if (__any_sync(0xffffffffu, active)) {
        for (int z = 0; z < TZ; ++z) {
          const R w3 = active ? wk3[z] : R(0);
          if (!__any_sync(0xffffffffu, w3 != R(0))) continue;
#pragma unroll
          for (int y = 0; y < TY; ++y) {
            const R w23 = w2[y] * w3;
            if (!__any_sync(0xffffffffu, w23 != R(0))) continue;
            R rs[NC];
#pragma unroll
            for (int c = 0; c < NC; ++c) rs[c] = R(0);
            const V* row = sG + (z * TY + y) * TX;
#pragma unroll
            for (int x = 0; x < TX; ++x) {
              const V g = row[x];
              const R w = w1[x];
              if constexpr (NC == 4) {
                rs[0] = fma(w, g.x, rs[0]);
                rs[1] = fma(w, g.y, rs[1]);
                rs[2] = fma(w, g.z, rs[2]);
                rs[3] = fma(w, g.w, rs[3]);
              } else {
                rs[0] = fma(w, g, rs[0]);
              }
            }
#pragma unroll
            for (int c = 0; c < NC; ++c) acc[c] += static_cast<double>(w23 * rs[c]);
          }
        }
      }
      if (active) {
        const int sidx = ((ps >> 16) * sd.S[1] + ((ps >> 8) & 0xff)) * sd.S[0] + (ps & 0xff);
        double* dst = part + (static_cast<size_t>(k) * nslots + sidx) * NC;
#pragma unroll
        for (int c = 0; c < NC; ++c) dst[c] = acc[c];
      }
      __syncthreads();
    }
  }
}

// Final per-atom sum of the slot partials in a fixed order, with the assembly
// of fft/ewald_fft_3d.f90:121-132: pot = (sr + lr) + self, force = sr + q lr.
template <int NC>
__global__ void k_gather_final(const int4* __restrict__ slot, const int* __restrict__ perm,
                               const double* __restrict__ part, int n, StencilDims sd,
                               const double* __restrict__ q, double self_coef,
                               const double* __restrict__ pot_sr, const double* __restrict__ f_sr,
                               double* __restrict__ pot, double* __restrict__ force) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int4 si = slot[k];
  const int cx = slot_count(si.x), cy = slot_count(si.y), cz = slot_count(si.z);
  const int nslots = sd.S[0] * sd.S[1] * sd.S[2];
  const double* pk = part + static_cast<size_t>(k) * nslots * NC;
  double acc[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) acc[c] = 0.0;
  for (int sz = 0; sz < cz; ++sz)
    for (int sy = 0; sy < cy; ++sy)
      for (int sx = 0; sx < cx; ++sx) {
        const double* pp = pk + ((sz * sd.S[1] + sy) * sd.S[0] + sx) * NC;
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[c] += pp[c];
      }
  const int i = perm[k];
  const double qi = q[i];
  pot[i] = (pot_sr[i] + acc[0]) + self_coef * qi;
  if (NC == 4 && force) {
#pragma unroll
    for (int d = 0; d < 3; ++d) force[3 * i + d] = f_sr[3 * i + d] + qi * acc[1 + d];
  }
}

}  // namespace

void launch_weights(const MeshPlan& mp, const int4* mc, const double4* fr, int n, void* wtab,
                    void* qk, int4* slot, cudaStream_t st) {
  if (n == 0) return;
  const int threads = 128, blocks = (3 * n + threads - 1) / threads;
  if (mp.mixed)
    k_weights_tiled<float><<<blocks, threads, 0, st>>>(mc, fr, n, mp.sd, static_cast<float*>(wtab),
                                                        static_cast<float*>(qk), slot);
  else
    k_weights_tiled<double><<<blocks, threads, 0, st>>>(mc, fr, n, mp.sd, static_cast<double*>(wtab),
                                                         static_cast<double*>(qk), slot);
  ++g_launches;
}

void launch_spread(const MeshPlan& mp, const int4* slot, const void* wtab, const void* qk,
                   const int* tile_start, void* grid, cudaStream_t st) {
  dim3 grd(mp.sd.ntiles[0], mp.sd.ntiles[1], mp.sd.ntiles[2]);
  if (mp.mixed)
    k_spread_tiles<float><<<grd, kThreads, 0, st>>>(slot, static_cast<const float*>(wtab),
                                                     static_cast<const float*>(qk), tile_start,
                                                     mp.tl[0], mp.tl[1], mp.tl[2], mp.sd,
                                                     static_cast<float*>(grid));
  else
    k_spread_tiles<double><<<grd, kThreads, 0, st>>>(slot, static_cast<const double*>(wtab),
                                                      static_cast<const double*>(qk), tile_start,
                                                      mp.tl[0], mp.tl[1], mp.tl[2], mp.sd,
                                                      static_cast<double*>(grid));
  ++g_launches;
}

void launch_gather(const MeshPlan& mp, const int4* slot, const void* wtab, const int* tile_start,
                   const void* grid, int nc, double* part, cudaStream_t st) {
  dim3 grd(mp.sd.ntiles[0], mp.sd.ntiles[1], mp.sd.ntiles[2]);
  const size_t pts = static_cast<size_t>(TX) * TY * TZ;
#define EWG_GATHER(R, NC)                                                                         \
  k_gather_tiles<R, NC><<<grd, kGatherThreads, pts * NC * sizeof(R), st>>>(                         \
      slot, static_cast<const R*>(wtab), tile_start, mp.tl[0], mp.tl[1], mp.tl[2], mp.sd,           \
      static_cast<const R*>(grid), part)
  if (mp.mixed) {
    if (nc == 4)
      EWG_GATHER(float, 4);
    else
      EWG_GATHER(float, 1);
  } else {
    if (nc == 4)
      EWG_GATHER(double, 4);
    else
      EWG_GATHER(double, 1);
  }
#undef EWG_GATHER
  ++g_launches;
}

int stencil_configure_kernels() {
  const int bytes = TX * TY * TZ * 4 * 8;
  cudaFuncSetAttribute(k_gather_tiles<double, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  cudaFuncSetAttribute(k_gather_tiles<double, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  cudaFuncSetAttribute(k_gather_tiles<float, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  cudaFuncSetAttribute(k_gather_tiles<float, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  return cudaGetLastError() == cudaSuccess ? EWG_OK : EWG_ERR_CUDA;
}

void launch_gather_final(const MeshPlan& mp, const int4* slot, const int* perm, const double* part,
                         int nc, int n, const double* q, double self_coef, const double* pot_sr,
                         const double* f_sr, double* pot, double* force, cudaStream_t st) {
  if (n == 0) return;
  const int threads = 128, blocks = (n + threads - 1) / threads;
  if (nc == 4)
    k_gather_final<4><<<blocks, threads, 0, st>>>(slot, perm, part, n, mp.sd, q, self_coef, pot_sr,
                                                   f_sr, pot, force);
  else
    k_gather_final<1><<<blocks, threads, 0, st>>>(slot, perm, part, n, mp.sd, q, self_coef, pot_sr,
                                                   f_sr, pot, nullptr);
  ++g_launches;
}

}  // namespace ewg
