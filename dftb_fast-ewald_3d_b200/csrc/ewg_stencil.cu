// ewg_stencil.cu -- the particle side of the NFFT: window weights, spread and
// gather (nfft/nfft.f90:122-159, :253-278, :380-402).
//
// Tiling.  The fine grid is cut into tiles of 8 x 8 x 8 points.  Along each
// axis an atom's stencil [c-m, c+m] (mod n) runs through at most S_d
// consecutive tiles starting at tile f_d; the atom meets every tile of that
// S_x x S_y x S_z block once ("slots").
//
// Weights.  Per atom and axis the window weights are stored already laid out
// per touched tile (S_d * 8 values; zero outside the stencil and beyond the
// grid end; points a wrapping stencil reaches twice carry the sum).  A kernel
// then reads an atom's weights for a tile with no index arithmetic.
//
// Pairs.  Once per geometry, every (atom, tile) pair is binned by tile with a
// counting sort whose buckets are ordered by atom index, so each tile owns an
// exact, deterministic list of the atoms that reach it.
//
// Spread: a CTA owns a tile and writes it once (no atomics, no zeroing, fixed
// order).  Both precision forms contract on the FP64 tensor cores (DMMA); the
// mixed form's FP32 weight rows are widened to FP64 as they are staged and its
// grid is written in FP32.  The FP32 CUDA-core spread (a kernel shape of the
// mixed form) keeps two x-pencils of 8 points per lane in registers and adds
// q w1 w2 w3 atom by atom in list order (groups of 16 atoms in FP32, the group
// sums in FP64).
// Gather: a CTA stages its tile in shared memory and contracts it with the
// weight rows of its atoms on the tensor cores (FP32 tiles widened as they are
// staged), or, on the FP32 CUDA cores, walks the tile's points in lockstep so
// every grid value is a shared-memory broadcast.  Each atom's partial goes to
// its slot for this tile; a final kernel sums each atom's slots in a fixed
// order.  Results are bitwise reproducible.

#include <cuda_runtime.h>

#include <climits>
#include <type_traits>

#include "ewg_kernels.h"

namespace ewg {

namespace {

constexpr int TX = kTileX, TY = kTileY, TZ = kTileZ;
constexpr int kSpreadLanes = TY * TZ / 2;  // FP32 spread: one warp, two x-pencils per lane
constexpr int kSpreadChunk = 64;   // atoms whose weights are staged at once
constexpr int kSpreadGroup = 16;   // FP32 spread: atoms summed in FP32 before the FP64 add
// Gather: atoms per lane and warps sharing one staged tile, per precision.
template <typename R>
struct GatherShape {
  static constexpr int atoms = 2;
  static constexpr int warps = sizeof(R) == 8 ? 1 : 2;
};

__device__ __forceinline__ int pmod(int a, int n) {
  int r = a % n;
  return r < 0 ? r + n : r;
}

// One tile row of eight weights, 16-byte aligned.
__device__ __forceinline__ void store_row(float* out, const float (&v)[8]) {
  reinterpret_cast<float4*>(out)[0] = make_float4(v[0], v[1], v[2], v[3]);
  reinterpret_cast<float4*>(out)[1] = make_float4(v[4], v[5], v[6], v[7]);
}
__device__ __forceinline__ void store_row(double* out, const double (&v)[8]) {
#pragma unroll
  for (int p = 0; p < 8; p += 2)
    reinterpret_cast<double2*>(out)[p / 2] = make_double2(v[p], v[p + 1]);
}

__device__ __forceinline__ int slot_first(int packed) { return packed & 0xffff; }
__device__ __forceinline__ int slot_count(int packed) { return packed >> 16; }

// ---------------------------------------------------------------------------
// Tiled window weights, one thread per (atom, axis, tile slot): eight points
// each, so an atom's S_x + S_y + S_z rows are computed in parallel.
// ---------------------------------------------------------------------------
// Row r (axis and slot) of sorted atom k.
template <typename R>
__device__ __forceinline__ void weights_row(const int4* __restrict__ mc,
                                            const double4* __restrict__ fr,
                                            const int* __restrict__ perm, int k, int r,
                                            const StencilDims& sd, R* __restrict__ wtab,
                                            R* __restrict__ qk, int4* __restrict__ slot) {
  const int d = r < sd.S[0] ? 0 : (r < sd.S[0] + sd.S[1] ? 1 : 2);
  const int s = r - (d == 0 ? 0 : (d == 1 ? sd.S[0] : sd.S[0] + sd.S[1]));
  const int i = perm[k];
  const int4 c4 = mc[i];
  const double4 f4 = fr[i];
  const int c = d == 0 ? c4.x : (d == 1 ? c4.y : c4.z);
  const double frac = d == 0 ? f4.x : (d == 1 ? f4.y : f4.z);
  const int nd = sd.n[d], T = sd.T[d], nt = sd.ntiles[d];
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
  R* out = wtab + static_cast<size_t>(k) * sd.wstride + sd.woff[d] + s * T;
  // Window derivative with respect to the atom's fractional coordinate s_d:
  // the point sits at u = o - frac grid units from the atom, and
  // d/ds_d [pref exp(-u^2 / b)] = n_d (2 u / b) pref exp(-u^2 / b).
  const double dscale = -2.0 * static_cast<double>(nd) / sd.b;
  const int origin = ((first + s) % nt) * T;
  R wv[TX], dv[TX];
  static_assert(TX == TY && TY == TZ, "one row length for all axes");
  if (2 * m + 1 < nd) {
    // Every point has at most one image in [-m, m]: the offsets of the row are
    // consecutive (one wrap at most) and the eight terms are independent.
    const int o0 = pmod(origin - c, nd);
#pragma unroll
    for (int p = 0; p < TX; ++p) {
      int o = o0 + p;
      if (o >= nd) o -= nd;
      if (o > m) o -= nd;  // largest offset <= m congruent to P - c
      const bool live = s < count && origin + p < nd && o >= -m;
      const double dd = frac - static_cast<double>(o);
      const double e = sd.pref * exp(-(dd * dd) / sd.b);
      wv[p] = static_cast<R>(live ? e : 0.0);
      dv[p] = static_cast<R>(live ? dscale * dd * e : 0.0);
    }
  } else {
#pragma unroll
    for (int p = 0; p < TX; ++p) {
      const int P = origin + p;
      double w = 0.0, dw = 0.0;
      if (s < count && P < nd) {
        int o = pmod(P - c, nd);  // largest offset <= m congruent to P - c
        while (o > m) o -= nd;
        while (o + nd <= m) o += nd;
        for (; o >= -m; o -= nd) {
          const double dd = frac - static_cast<double>(o);
          const double e = sd.pref * exp(-(dd * dd) / sd.b);
          w += e;
          dw += dscale * dd * e;
        }
      }
      wv[p] = static_cast<R>(w);
      dv[p] = static_cast<R>(dw);
    }
  }
  // Rows start on multiples of eight values: whole 16-byte stores.
  store_row(out, wv);
  if (sd.ad) store_row(out + sd.dwoff, dv);
  if (s != 0) return;  // the axis' first slot thread writes the slot record
  int* sp = reinterpret_cast<int*>(&slot[k]);
  sp[d] = first | (count << 16);
  if (d == 0) {
    sp[3] = 0;
    qk[k] = static_cast<R>(f4.w);
  }
}

template <typename R>
__global__ void k_weights_tiled(const int4* __restrict__ mc, const double4* __restrict__ fr,
                                const int* __restrict__ perm, int n, StencilDims sd,
                                R* __restrict__ wtab, R* __restrict__ qk,
                                int4* __restrict__ slot) {
  chain_enter();
  const int SS = sd.S[0] + sd.S[1] + sd.S[2];
  const long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= static_cast<long>(SS) * n) return;
  const int k = static_cast<int>(idx / SS);
  weights_row<R>(mc, fr, perm, k, static_cast<int>(idx - static_cast<long>(k) * SS), sd, wtab, qk,
                 slot);
}

// Every cell of a batch: item idx is (atom, row) of its cell (prefix over the
// cells' natoms (S_x + S_y + S_z)); the weight rows keep the batch's common
// per-atom stride.
template <typename R>
__global__ void k_weights_seg(const BatchCell* __restrict__ cells, const int* __restrict__ prefix,
                              int ncells, long nitems, const int4* __restrict__ mc,
                              const double4* __restrict__ fr, const int* __restrict__ perm,
                              R* __restrict__ wtab, R* __restrict__ qk, int4* __restrict__ slot) {
  chain_enter();
  const long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= nitems) return;
  const int c = seg_cell(prefix, ncells, idx);
  const BatchCell& bc = cells[c];
  const StencilDims sd = bc.sd;
  const int SS = sd.S[0] + sd.S[1] + sd.S[2];
  const int local = static_cast<int>(idx - prefix[c]);
  const int kl = local / SS;
  weights_row<R>(mc, fr, perm, bc.atom0 + kl, local - kl * SS, sd, wtab, qk, slot);
}

// ---------------------------------------------------------------------------
// (atom, tile) pair binning.
// ---------------------------------------------------------------------------
template <class F>
__device__ __forceinline__ void for_each_tile(const int4& si, const StencilDims& sd, F f) {
  const int cx = slot_count(si.x), cy = slot_count(si.y), cz = slot_count(si.z);
  const int fx = slot_first(si.x), fy = slot_first(si.y), fz = slot_first(si.z);
  for (int sz = 0; sz < cz; ++sz) {
    const int tz = (fz + sz) % sd.ntiles[2];
    for (int sy = 0; sy < cy; ++sy) {
      const int ty = (fy + sy) % sd.ntiles[1];
      for (int sx = 0; sx < cx; ++sx) {
        const int tx = (fx + sx) % sd.ntiles[0];
        f((tz * sd.ntiles[1] + ty) * sd.ntiles[0] + tx, sx | (sy << 8) | (sz << 16));
      }
    }
  }
}

// One thread per (atom, slot of the S_x x S_y x S_z block); slots past the
// atom's own tile counts are skipped.
// Slot s of sorted atom k: its tile (the cell's own numbering) and packed
// slot, false for slots past the atom's tile counts.
__device__ __forceinline__ bool pair_of(const int4* __restrict__ slot, int k, int s,
                                        const StencilDims& sd, int* tile, int* packed) {
  const int sx = s % sd.S[0], sy = (s / sd.S[0]) % sd.S[1], sz = s / (sd.S[0] * sd.S[1]);
  const int4 si = slot[k];
  if (sx >= slot_count(si.x) || sy >= slot_count(si.y) || sz >= slot_count(si.z)) return false;
  const int tx = (slot_first(si.x) + sx) % sd.ntiles[0];
  const int ty = (slot_first(si.y) + sy) % sd.ntiles[1];
  const int tz = (slot_first(si.z) + sz) % sd.ntiles[2];
  *tile = (tz * sd.ntiles[1] + ty) * sd.ntiles[0] + tx;
  *packed = sx | (sy << 8) | (sz << 16);
  return true;
}

// Item idx of a batch's (atom, slot) launch: its cell, sorted atom, tile
// (global numbering: the cell's tile0 added) and packed slot.
__device__ __forceinline__ bool pair_of_seg(const BatchCell* __restrict__ cells,
                                            const int* __restrict__ prefix, int ncells, long idx,
                                            const int4* __restrict__ slot, int* tile, int* k,
                                            int* packed) {
  const int c = seg_cell(prefix, ncells, idx);
  const BatchCell& bc = cells[c];
  const int S = bc.sd.S[0] * bc.sd.S[1] * bc.sd.S[2];
  const int local = static_cast<int>(idx - prefix[c]);
  const int kl = local / S;
  *k = bc.atom0 + kl;
  const StencilDims sd = bc.sd;
  if (!pair_of(slot, *k, local - kl * S, sd, tile, packed)) return false;
  *tile += bc.tile0;
  return true;
}

__global__ void k_pair_count_seg(const BatchCell* __restrict__ cells,
                                 const int* __restrict__ prefix, int ncells, long nitems,
                                 const int4* __restrict__ slot, int* __restrict__ counts) {
  const long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  int tile, k, packed;
  if (idx < nitems && pair_of_seg(cells, prefix, ncells, idx, slot, &tile, &k, &packed))
    atomicAdd(&counts[tile], 1);
}

__global__ void k_pair_scatter_seg(const BatchCell* __restrict__ cells,
                                   const int* __restrict__ prefix, int ncells, long nitems,
                                   const int4* __restrict__ slot, const int* __restrict__ starts,
                                   int* __restrict__ cursor, int2* __restrict__ tmp) {
  chain_enter();
  const long idx = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  int tile, k, packed;
  if (idx < nitems && pair_of_seg(cells, prefix, ncells, idx, slot, &tile, &k, &packed))
    tmp[starts[tile] + atomicAdd(&cursor[tile], 1)] = make_int2(k, packed);
}

// As k_pair_rank, the entry's cell found from its atom (sorted ranges follow
// the cells' atom ranges).
__global__ void k_pair_rank_seg(const BatchCell* __restrict__ cells,
                                const int* __restrict__ atom_prefix, int ncells,
                                const int2* __restrict__ tmp, const int* __restrict__ starts,
                                int ntiles, const int4* __restrict__ slot,
                                int2* __restrict__ pairs) {
  chain_enter();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= starts[ntiles]) return;
  const int2 v = tmp[e];
  const BatchCell& bc = cells[seg_cell(atom_prefix, ncells, v.x)];
  const int4 si = slot[v.x];
  const int tx = (slot_first(si.x) + (v.y & 0xff)) % bc.sd.ntiles[0];
  const int ty = (slot_first(si.y) + ((v.y >> 8) & 0xff)) % bc.sd.ntiles[1];
  const int tz = (slot_first(si.z) + (v.y >> 16)) % bc.sd.ntiles[2];
  const int tile = bc.tile0 + (tz * bc.sd.ntiles[1] + ty) * bc.sd.ntiles[0] + tx;
  const int b = starts[tile], end = starts[tile + 1];
  int r = 0;
  for (int j = b; j < end; ++j) r += tmp[j].x < v.x;
  pairs[b + r] = v;
}

__device__ __forceinline__ bool pair_of_thread(const int4* __restrict__ slot, int n,
                                               const StencilDims& sd, int* tile, int* k,
                                               int* packed) {
  const int S = sd.S[0] * sd.S[1] * sd.S[2];
  const long t = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<long>(n) * S) return false;
  *k = static_cast<int>(t / S);
  const int s = static_cast<int>(t - static_cast<long>(*k) * S);
  return pair_of(slot, *k, s, sd, tile, packed);
}

__global__ void k_pair_count(const int4* __restrict__ slot, int n, StencilDims sd,
                             int* __restrict__ counts) {
  int tile, k, packed;
  if (pair_of_thread(slot, n, sd, &tile, &k, &packed)) atomicAdd(&counts[tile], 1);
}

__global__ void k_pair_scatter(const int4* __restrict__ slot, int n, StencilDims sd,
                               const int* __restrict__ starts, int* __restrict__ cursor,
                               int2* __restrict__ tmp) {
  chain_enter();
  int tile, k, packed;
  if (pair_of_thread(slot, n, sd, &tile, &k, &packed))
    tmp[starts[tile] + atomicAdd(&cursor[tile], 1)] = make_int2(k, packed);
}

// One thread per entry: orders each tile's bucket by atom index (atoms are
// unique within a bucket) by counting the bucket's entries with a smaller atom.
// The entry's tile follows from its atom's slot record and its packed slot.
__global__ void k_pair_rank(const int2* __restrict__ tmp, const int* __restrict__ starts,
                            int ntiles, const int4* __restrict__ slot, StencilDims sd,
                            int2* __restrict__ pairs) {
  chain_enter();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= starts[ntiles]) return;
  const int2 v = tmp[e];
  const int4 si = slot[v.x];
  const int tx = (slot_first(si.x) + (v.y & 0xff)) % sd.ntiles[0];
  const int ty = (slot_first(si.y) + ((v.y >> 8) & 0xff)) % sd.ntiles[1];
  const int tz = (slot_first(si.z) + (v.y >> 16)) % sd.ntiles[2];
  const int tile = (tz * sd.ntiles[1] + ty) * sd.ntiles[0] + tx;
  const int b = starts[tile], end = starts[tile + 1];
  int r = 0;
  for (int j = b; j < end; ++j) r += tmp[j].x < v.x;
  pairs[b + r] = v;
}

// Eight consecutive FP32 weights (32 B; every per-tile weight row starts on
// such a boundary) with vector loads.
__device__ __forceinline__ void load8(const float* __restrict__ p, float* out) {
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const float4 v = reinterpret_cast<const float4*>(p)[i];
    out[4 * i] = v.x;
    out[4 * i + 1] = v.y;
    out[4 * i + 2] = v.z;
    out[4 * i + 3] = v.w;
  }
}

// ---------------------------------------------------------------------------
// Spread
// ---------------------------------------------------------------------------
// FP32 form: one warp per tile; each lane owns two x-pencils, (py, pz) and
// (py + 4, pz), so every pair of shared-memory reads of an atom's x weights
// feeds 16 multiply-adds.
template <typename R>
__device__ __forceinline__ void spread_tiles_body(int tx, int ty, int tz,
                                                  const int* __restrict__ tile_start,
                                                               const int2* __restrict__ pairs,
                                                               const R* __restrict__ wtab,
                                                               const R* __restrict__ qk,
                                                               StencilDims sd, R* __restrict__ grid) {
  chain_enter();
  __shared__ R sW1[kSpreadChunk][TX];
  __shared__ R sW2[kSpreadChunk][TY];
  __shared__ R sW3[kSpreadChunk][TZ];
  const int tile = (tz * sd.ntiles[1] + ty) * sd.ntiles[0] + tx;
  const int x0 = tx * TX, y0 = ty * TY, z0 = tz * TZ;
  const int py = threadIdx.x % (TY / 2), pz = threadIdx.x / (TY / 2);
  double acc[2][TX];
#pragma unroll
  for (int x = 0; x < TX; ++x) acc[0][x] = acc[1][x] = 0.0;
  const int p0 = tile_start[tile], p1 = tile_start[tile + 1];
  for (int b0 = p0; b0 < p1; b0 += kSpreadChunk) {
    const int nb = min(kSpreadChunk, p1 - b0);
    __syncthreads();  // the previous chunk's weights are no longer read
    // Each lane stages whole atoms of the chunk: its pair, charge and the
    // 3 x 8 weights for this tile, in independent vector loads.
    for (int a = threadIdx.x; a < nb; a += kSpreadLanes) {
      const int2 pr = pairs[b0 + a];
      const R* wk = wtab + static_cast<size_t>(pr.x) * sd.wstride;
      R t1[TX], t2[TY], t3[TZ];
      load8(wk + sd.woff[0] + (pr.y & 0xff) * TX, t1);
      load8(wk + sd.woff[1] + ((pr.y >> 8) & 0xff) * TY, t2);
      load8(wk + sd.woff[2] + (pr.y >> 16) * TZ, t3);
      const R qa = qk[pr.x];
#pragma unroll
      for (int x = 0; x < TX; ++x) sW1[a][x] = t1[x];
#pragma unroll
      for (int y = 0; y < TY; ++y) sW2[a][y] = t2[y];
#pragma unroll
      for (int z = 0; z < TZ; ++z) sW3[a][z] = t3[z] * qa;
    }
    __syncthreads();
    // Groups of kSpreadGroup atoms are summed in R, each group sum then
    // added to the FP64 pencil: one FP32 -> FP64 conversion per point and
    // group instead of per point and atom (the conversions, not the
    // multiply-adds, bounded the FP32 form).
    for (int g0 = 0; g0 < nb; g0 += kSpreadGroup) {
      const int g1 = min(g0 + kSpreadGroup, nb);
      R part[2][TX];
#pragma unroll
      for (int x = 0; x < TX; ++x) part[0][x] = part[1][x] = R(0);
      for (int a = g0; a < g1; ++a) {
        const R w3 = sW3[a][pz];
        const R s0 = sW2[a][py] * w3, s1 = sW2[a][py + TY / 2] * w3;
#pragma unroll
        for (int x = 0; x < TX; ++x) {
          const R w1 = sW1[a][x];
          part[0][x] = fma(s0, w1, part[0][x]);
          part[1][x] = fma(s1, w1, part[1][x]);
        }
      }
#pragma unroll
      for (int x = 0; x < TX; ++x) {
        acc[0][x] += static_cast<double>(part[0][x]);
        acc[1][x] += static_cast<double>(part[1][x]);
      }
    }
  }
  const int ex = min(TX, sd.n[0] - x0), ey = min(TY, sd.n[1] - y0), ez = min(TZ, sd.n[2] - z0);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int y = py + h * (TY / 2);
    if (y < ey && pz < ez) {
      R* row = grid + (static_cast<size_t>(z0 + pz) * sd.n[1] + y0 + y) * sd.n[0] + x0;
#pragma unroll
      for (int x = 0; x < TX; ++x)
        if (x < ex) row[x] = static_cast<R>(acc[h][x]);
    }
  }
}

// ---------------------------------------------------------------------------
// FP64 spread on the tensor cores.  For each z-plane of the tile the spread is
// a sum of rank-one products, G_z[y][x] = sum_a (q_a w3_a(z) w2_a(y)) w1_a(x),
// i.e. the 8 x 8 matrix product U_z W1 with U_z[y][a] = q_a w3_a(z) w2_a(y) and
// W1[a][x] = w1_a(x).  A CTA owns a tile and accumulates its eight planes
// with DMMA (mma.sync m8n8k4, FP64 in and out, IEEE fused multiply-adds), four
// atoms per step, in list order: deterministic, no atomics.
// Fragment layouts (m8n8k4, .row.col): A[y][k] at lane 4y + k, B[k][x] at lane
// 4x + k, C[y][x] at lane 4y + x/2 (element x mod 2).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma_m8n8k4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

constexpr int kGatherWarps = 4;   // tensor-core i k gather: warps per tile
constexpr int kGatherMB = 2;      // tensor-core i k gather: M blocks of 8 atoms per warp and round
constexpr int kGatherAdWarps = 2;  // tensor-core gather with window derivatives: warps per tile
// FP32 CUDA-core gather with window derivatives: one atom per lane (74 registers, so
// about 13 CTAs per SM) and two warps per tile.
constexpr int kGatherAdF32Atoms = 1, kGatherAdF32Warps = 2;
constexpr int kSpreadAtoms = 32;  // tensor-core spread: atoms staged per round, one per lane
constexpr int kWRow = 12;         // doubles per staged weight row: 8 used; the
                                  // padding makes the fragment reads conflict-free

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Two consecutive elements from global into shared memory as doubles: a
// 16-byte cp.async for FP64 data; for the mixed form's FP32 tiles and weight
// rows an 8-byte load widened to FP64, so the same DMMA code contracts them.
__device__ __forceinline__ void stage2(double* dst, const double* src) { cp_async16(dst, src); }
__device__ __forceinline__ void stage2(double* dst, const float* src) {
  const float2 v = __ldg(reinterpret_cast<const float2*>(src));
  dst[0] = v.x;
  dst[1] = v.y;
}

// One warp per tile owning all eight z-planes, so each step's x and y weights
// are read from shared memory once for the eight planes; the lanes stage up to
// 32 atoms' weight rows per round with asynchronous 16-byte copies.
template <typename R>
__device__ __forceinline__ void spread_tiles_dmma_body(int tx, int ty, int tz,
                                                       const int* __restrict__ tile_start,
                                                       const int2* __restrict__ pairs,
                                                       const R* __restrict__ wtab,
                                                       const R* __restrict__ qk, StencilDims sd,
                                                       R* __restrict__ grid) {
  chain_enter();
  __shared__ __align__(16) double sW[3][kSpreadAtoms][kWRow];
  __shared__ double sQ[kSpreadAtoms];
  const int tile = (tz * sd.ntiles[1] + ty) * sd.ntiles[0] + tx;
  const int x0 = tx * TX, y0 = ty * TY, z0 = tz * TZ;
  const int lane = threadIdx.x;
  const int fr = lane >> 2, fk = lane & 3;  // fragment row (y, or x for B) and k
  double acc[TZ][2];
#pragma unroll
  for (int z = 0; z < TZ; ++z) acc[z][0] = acc[z][1] = 0.0;
  const int p0 = tile_start[tile], p1 = tile_start[tile + 1];
  for (int b0 = p0; b0 < p1; b0 += kSpreadAtoms) {
    const int nb = min(kSpreadAtoms, p1 - b0);
    __syncwarp();  // the previous round's weights are no longer read
    const int a = lane;
    if (a < nb) {
      const int2 pr = pairs[b0 + a];
      const R* wk = wtab + static_cast<size_t>(pr.x) * sd.wstride;
      const R* src[3] = {wk + sd.woff[0] + (pr.y & 0xff) * TX,
                         wk + sd.woff[1] + ((pr.y >> 8) & 0xff) * TY,
                         wk + sd.woff[2] + (pr.y >> 16) * TZ};
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int j = 0; j < 4; ++j) stage2(&sW[d][a][2 * j], src[d] + 2 * j);
      sQ[a] = qk[pr.x];
    } else if (a < ((nb + 3) & ~3)) {  // padding atoms of the last group of four
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int j = 0; j < 8; ++j) sW[d][a][j] = 0.0;
      sQ[a] = 0.0;
    }
    cp_async_wait_all();
    __syncwarp();
    for (int k0 = 0; k0 < nb; k0 += 4) {
      const int aa = k0 + fk;
      const double bw = sW[0][aa][fr];            // B[k][x = fr]
      const double w2q = sW[1][aa][fr] * sQ[aa];  // A[y = fr][k] = q w2(y) w3(z)
#pragma unroll
      for (int z = 0; z < TZ; ++z) dmma_m8n8k4(acc[z][0], acc[z][1], w2q * sW[2][aa][z], bw);
    }
  }
  const int ex = min(TX, sd.n[0] - x0), ey = min(TY, sd.n[1] - y0), ez = min(TZ, sd.n[2] - z0);
  const int y = fr, x = 2 * fk;
  if (y < ey) {
#pragma unroll
    for (int z = 0; z < TZ; ++z) {
      if (z >= ez) break;
      R* row = grid + (static_cast<size_t>(z0 + z) * sd.n[1] + y0 + y) * sd.n[0] + x0 + x;
      if (x + 1 < ex) {
        row[0] = static_cast<R>(acc[z][0]);
        row[1] = static_cast<R>(acc[z][1]);
      } else if (x < ex) {
        row[0] = static_cast<R>(acc[z][0]);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Gather.  One warp per CTA; each lane carries A atoms of the tile's list, so
// every grid value read from shared memory (a broadcast: all lanes read the
// same point) feeds A atoms.
// ---------------------------------------------------------------------------
template <typename R, int NC, int A, int WARPS>
__device__ __forceinline__ void gather_tiles_body(int tx, int ty, int tz,
                                                  const int* __restrict__ tile_start,
                                                             const int2* __restrict__ pairs,
                                                             const R* __restrict__ wtab,
                                                             StencilDims sd,
                                                             const R* __restrict__ grid,
                                                             double* __restrict__ part) {
  chain_enter();
  using V = typename std::conditional<
      NC == 4, typename std::conditional<sizeof(R) == 8, double4, float4>::type, R>::type;
  __shared__ V sG[TZ * TY * TX];
  __shared__ R sW3[WARPS][TZ][32 * A];  // z weights, lane fastest
  const int tile = (tz * sd.ntiles[1] + ty) * sd.ntiles[0] + tx;
  const int x0 = tx * TX, y0 = ty * TY, z0 = tz * TZ;
  const int ex = min(TX, sd.n[0] - x0), ey = min(TY, sd.n[1] - y0), ez = min(TZ, sd.n[2] - z0);
  const int p0 = tile_start[tile], p1 = tile_start[tile + 1];
  if (p0 == p1) return;  // no atom reaches this tile
#pragma unroll 4
  for (int t = threadIdx.x; t < TX * TY * TZ; t += 32 * WARPS) {
    const int x = t % TX, y = (t / TX) % TY, z = t / (TX * TY);
    V v;
    if (x < ex && y < ey && z < ez) {
      v = reinterpret_cast<const V*>(grid)[(static_cast<size_t>(z0 + z) * sd.n[1] + y0 + y) * sd.n[0] +
                                           x0 + x];
    } else {
      if constexpr (NC == 4)
        v = V{R(0), R(0), R(0), R(0)};
      else
        v = R(0);
    }
    sG[t] = v;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nslots = sd.pstride;
  for (int a0 = p0 + warp * 32 * A; a0 < p1; a0 += WARPS * 32 * A) {
    R w1[A][TX], w2[A][TY];
    int2 pr[A];
    bool act[A];
#pragma unroll
    for (int a = 0; a < A; ++a) {
      const int e = a0 + a * 32 + lane;
      act[a] = e < p1;
      pr[a] = act[a] ? pairs[e] : make_int2(0, 0);
      const R* wk = wtab + static_cast<size_t>(pr[a].x) * sd.wstride;
#pragma unroll
      for (int x = 0; x < TX; ++x) w1[a][x] = act[a] ? wk[sd.woff[0] + (pr[a].y & 0xff) * TX + x] : R(0);
#pragma unroll
      for (int y = 0; y < TY; ++y)
        w2[a][y] = act[a] ? wk[sd.woff[1] + ((pr[a].y >> 8) & 0xff) * TY + y] : R(0);
      const R* wz = wk + sd.woff[2] + (pr[a].y >> 16) * TZ;
#pragma unroll
      for (int z = 0; z < TZ; ++z) sW3[warp][z][a * 32 + lane] = act[a] ? wz[z] : R(0);
    }
    __syncwarp();
    double acc[A][NC];
#pragma unroll
    for (int a = 0; a < A; ++a)
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[a][c] = 0.0;
#pragma unroll 1
    for (int z = 0; z < TZ; ++z) {
      R w3[A];
#pragma unroll
      for (int a = 0; a < A; ++a) w3[a] = sW3[warp][z][a * 32 + lane];
      // The plane's rows are summed in R, the plane sum then added in FP64.
      R pl[A][NC];
#pragma unroll
      for (int a = 0; a < A; ++a)
#pragma unroll
        for (int c = 0; c < NC; ++c) pl[a][c] = R(0);
#pragma unroll
      for (int y = 0; y < TY; ++y) {
        R w23[A];
        bool any = false;
#pragma unroll
        for (int a = 0; a < A; ++a) {
          w23[a] = w2[a][y] * w3[a];
          any = any || (w23[a] != R(0));
        }
        if (!__any_sync(0xffffffffu, any)) continue;
        R rs[A][NC];
#pragma unroll
        for (int a = 0; a < A; ++a)
#pragma unroll
          for (int c = 0; c < NC; ++c) rs[a][c] = R(0);
        const V* row = sG + (z * TY + y) * TX;
#pragma unroll
        for (int x = 0; x < TX; ++x) {
          const V g = row[x];
#pragma unroll
          for (int a = 0; a < A; ++a) {
            if constexpr (NC == 4) {
              rs[a][0] = fma(w1[a][x], g.x, rs[a][0]);
              rs[a][1] = fma(w1[a][x], g.y, rs[a][1]);
              rs[a][2] = fma(w1[a][x], g.z, rs[a][2]);
              rs[a][3] = fma(w1[a][x], g.w, rs[a][3]);
            } else {
              rs[a][0] = fma(w1[a][x], g, rs[a][0]);
            }
          }
        }
#pragma unroll
        for (int a = 0; a < A; ++a)
#pragma unroll
          for (int c = 0; c < NC; ++c) pl[a][c] = fma(w23[a], rs[a][c], pl[a][c]);
      }
#pragma unroll
      for (int a = 0; a < A; ++a)
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[a][c] += static_cast<double>(pl[a][c]);
    }
#pragma unroll
    for (int a = 0; a < A; ++a) {
      if (!act[a]) continue;
      const int ps = pr[a].y;
      const int sidx = ((ps >> 16) * sd.S[1] + ((ps >> 8) & 0xff)) * sd.S[0] + (ps & 0xff);
      double* dst = part + (static_cast<size_t>(pr[a].x) * nslots + sidx) * NC;
#pragma unroll
      for (int c = 0; c < NC; ++c) dst[c] = acc[a][c];
    }
    __syncwarp();  // sW3 is rewritten by the next iteration
  }
}

// ---------------------------------------------------------------------------
// FP32 gather with window derivatives (force scheme ad).  The tile holds the
// potential grid g alone.  With W = w1 w2 w3 and D_d the same product with
// axis d's weights replaced by their derivatives with respect to s_d, an atom
// needs phi = sum W g and D_d = sum D_d g.  The derivative weights change sign
// across the stencil while g carries a large smooth part, so in FP32 the sums
// would cancel; they run instead on g' = g - c, with c the grid value at the
// tile's first point (subtracted once, when the tile is staged), and the
// tile's c terms are added back in FP64 from the tile's weight sums:
//   phi_t = sum_t W g' + c Sx Sy Sz,  D_1,t = sum_t dW_1 g' + c dSx Sy Sz, ...
// (S, dS: sums over the tile's points of the weights and their derivatives).
// Per (z, y) row two x sums, r0 = sum_x w1 g' and r1 = sum_x dw1 g', feed all
// four:  phi += w2 w3 r0, D_1 += w2 w3 r1, D_2 += dw2 w3 r0, D_3 += w2 dw3 r0.
// Lanes carry A atoms of the tile's list as in k_gather_tiles (x weights in
// registers, y and z rows staged in shared memory); products and plane sums in
// FP32, the sum over planes in FP64; the four partials go to the atom's slot.
// ---------------------------------------------------------------------------
template <int A, int WARPS>
__device__ __forceinline__ void gather_tiles_ad_body(int tx, int ty, int tz,
                                                     const int* __restrict__ tile_start,
                                                                const int2* __restrict__ pairs,
                                                                const float* __restrict__ wtab,
                                                                StencilDims sd,
                                                                const float* __restrict__ grid,
                                                                double* __restrict__ part) {
  chain_enter();
  __shared__ float sG[TZ * TY * TX];
  // y and z weights and their derivatives, lane fastest: [kind][row][lane]
  // with kind 0 = w2, 1 = dw2, 2 = w3, 3 = dw3.
  __shared__ float sYZ[WARPS][4][TY][32 * A];
  static_assert(TY == TZ, "y and z rows share one staging layout");
  const int tile = (tz * sd.ntiles[1] + ty) * sd.ntiles[0] + tx;
  const int x0 = tx * TX, y0 = ty * TY, z0 = tz * TZ;
  const int ex = min(TX, sd.n[0] - x0), ey = min(TY, sd.n[1] - y0), ez = min(TZ, sd.n[2] - z0);
  const int p0 = tile_start[tile], p1 = tile_start[tile + 1];
  if (p0 == p1) return;  // no atom reaches this tile
  const float cg = grid[(static_cast<size_t>(z0) * sd.n[1] + y0) * sd.n[0] + x0];
#pragma unroll 4
  for (int t = threadIdx.x; t < TX * TY * TZ; t += 32 * WARPS) {
    const int x = t % TX, y = (t / TX) % TY, z = t / (TX * TY);
    // points past the grid's end carry zero weight for every atom
    sG[t] = (x < ex && y < ey && z < ez)
                ? grid[(static_cast<size_t>(z0 + z) * sd.n[1] + y0 + y) * sd.n[0] + x0 + x] - cg
                : 0.0f;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nslots = sd.pstride;
  float(*YZ)[TY][32 * A] = sYZ[warp];
  for (int a0 = p0 + warp * 32 * A; a0 < p1; a0 += WARPS * 32 * A) {
    float w1[A][TX], d1[A][TX];
    int2 pr[A];
    bool act[A];
#pragma unroll
    for (int a = 0; a < A; ++a) {
      const int e = a0 + a * 32 + lane;
      act[a] = e < p1;
      pr[a] = act[a] ? pairs[e] : make_int2(0, 0);
      const float* wk = wtab + static_cast<size_t>(pr[a].x) * sd.wstride;
      const int ox = sd.woff[0] + (pr[a].y & 0xff) * TX;
      const int oy = sd.woff[1] + ((pr[a].y >> 8) & 0xff) * TY;
      const int oz = sd.woff[2] + (pr[a].y >> 16) * TZ;
      float t[4][8];
      if (act[a]) {
        load8(wk + ox, w1[a]);
        load8(wk + sd.dwoff + ox, d1[a]);
        load8(wk + oy, t[0]);
        load8(wk + sd.dwoff + oy, t[1]);
        load8(wk + oz, t[2]);
        load8(wk + sd.dwoff + oz, t[3]);
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) w1[a][j] = d1[a][j] = t[0][j] = t[1][j] = t[2][j] = t[3][j] = 0.0f;
      }
#pragma unroll
      for (int kd = 0; kd < 4; ++kd)
#pragma unroll
        for (int j = 0; j < 8; ++j) YZ[kd][j][a * 32 + lane] = t[kd][j];
    }
    __syncwarp();
    double acc[A][4];
    float sz[A], dsz[A];
#pragma unroll
    for (int a = 0; a < A; ++a) {
      sz[a] = dsz[a] = 0.0f;
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][c] = 0.0;
    }
#pragma unroll 1
    for (int z = 0; z < TZ; ++z) {
      float w3[A], d3[A], pl[A][4];
#pragma unroll
      for (int a = 0; a < A; ++a) {
        w3[a] = YZ[2][z][a * 32 + lane];
        d3[a] = YZ[3][z][a * 32 + lane];
        sz[a] += w3[a];
        dsz[a] += d3[a];
        pl[a][0] = pl[a][1] = pl[a][2] = pl[a][3] = 0.0f;  // plane sums, FP32
      }
#pragma unroll
      for (int y = 0; y < TY; ++y) {
        // A zero window product means the row lies outside the atom's stencil
        // along y or z, where the derivatives vanish as well.
        float w2[A], d2[A], w23[A];
        bool any = false;
#pragma unroll
        for (int a = 0; a < A; ++a) {
          w2[a] = YZ[0][y][a * 32 + lane];
          d2[a] = YZ[1][y][a * 32 + lane];
          w23[a] = w2[a] * w3[a];
          any = any || (w23[a] != 0.0f);
        }
        if (!__any_sync(0xffffffffu, any)) continue;
        float r0[A], r1[A];
#pragma unroll
        for (int a = 0; a < A; ++a) r0[a] = r1[a] = 0.0f;
        const float* row = sG + (z * TY + y) * TX;
#pragma unroll
        for (int x = 0; x < TX; ++x) {
          const float g = row[x];
#pragma unroll
          for (int a = 0; a < A; ++a) {
            r0[a] = fmaf(w1[a][x], g, r0[a]);
            r1[a] = fmaf(d1[a][x], g, r1[a]);
          }
        }
#pragma unroll
        for (int a = 0; a < A; ++a) {
          pl[a][0] = fmaf(w23[a], r0[a], pl[a][0]);
          pl[a][1] = fmaf(w23[a], r1[a], pl[a][1]);
          pl[a][2] = fmaf(d2[a] * w3[a], r0[a], pl[a][2]);
          pl[a][3] = fmaf(w2[a] * d3[a], r0[a], pl[a][3]);
        }
      }
#pragma unroll
      for (int a = 0; a < A; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][c] += static_cast<double>(pl[a][c]);
    }
#pragma unroll
    for (int a = 0; a < A; ++a) {
      if (!act[a]) continue;
      // the c terms of this tile: c (S or dS along each axis)
      double sx = 0.0, dsx = 0.0, sy = 0.0, dsy = 0.0;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        sx += w1[a][j];
        dsx += d1[a][j];
        sy += YZ[0][j][a * 32 + lane];
        dsy += YZ[1][j][a * 32 + lane];
      }
      const double c = cg;
      acc[a][0] += c * sx * sy * sz[a];
      acc[a][1] += c * dsx * sy * sz[a];
      acc[a][2] += c * sx * dsy * sz[a];
      acc[a][3] += c * sx * sy * dsz[a];
      const int ps = pr[a].y;
      const int sidx = ((ps >> 16) * sd.S[1] + ((ps >> 8) & 0xff)) * sd.S[0] + (ps & 0xff);
      double* dst = part + (static_cast<size_t>(pr[a].x) * nslots + sidx) * 4;
#pragma unroll
      for (int c4 = 0; c4 < 4; ++c4) dst[c4] = acc[a][c4];
    }
    __syncwarp();  // the staged rows are rewritten by the next iteration
  }
}

// ---------------------------------------------------------------------------
// FP64 gather on the tensor cores.  With the tile's values G[z][y][x][c] in
// shared memory, an atom's result is
//   phi_a,c = sum_z w3_a(z) sum_y w2_a(y) T_a[z][y][c],
//   T_a[z][y][c] = sum_x w1_a(x) G[z][y][x][c],
// and T is a matrix product: rows are atoms (M blocks of 8), the contraction
// runs over x (two k-steps of 4), columns over (c, y) (N blocks of the 8 y
// values of one component).  Scaling the A fragment by w3_a(z) lets the DMMA
// accumulators sum over the planes too.  Each warp takes up to MB M blocks of
// a round of 8 MB WARPS atoms; per plane and component it issues two DMMAs per M block.
// At the end the lane holding C for (atom, y pair) folds in w2, and the four
// lanes of an atom are summed with shuffles in a fixed order.  Partials go to the (atom, slot) array as in the CUDA-core
// gather; results are deterministic.
// Tile layout in shared memory: row (z, y) holds 8 points x NC values, padded
// to kGRow doubles so the B-fragment reads are nearly conflict-free.
// ---------------------------------------------------------------------------
template <int NC>
struct GatherRow {
  static constexpr int value = NC == 4 ? 34 : 12;  // 16-byte multiples
};
// WARPS warps per CTA, MB M blocks of 8 atoms per warp and round.
template <typename R, int NC, int WARPS, int MB>
__device__ __forceinline__ void gather_tiles_dmma_body(int tx, int ty, int tz,
                                                       const int* __restrict__ tile_start,
                                                       const int2* __restrict__ pairs,
                                                       const R* __restrict__ wtab, StencilDims sd,
                                                       const R* __restrict__ grid,
                                                       double* __restrict__ part) {
  chain_enter();
  constexpr int RS = GatherRow<NC>::value;
  constexpr int kGatherAtoms = WARPS * MB * 8;  // atoms staged per round
  __shared__ __align__(16) double sG[TZ * TY * RS];
  __shared__ __align__(16) double sW[3][kGatherAtoms][kWRow];
  __shared__ int2 sPair[kGatherAtoms];
  const int tile = (tz * sd.ntiles[1] + ty) * sd.ntiles[0] + tx;
  const int p0 = tile_start[tile], p1 = tile_start[tile + 1];
  if (p0 == p1) return;  // no atom reaches this tile
  const int x0 = tx * TX, y0 = ty * TY, z0 = tz * TZ;
  const int ex = min(TX, sd.n[0] - x0), ey = min(TY, sd.n[1] - y0), ez = min(TZ, sd.n[2] - z0);
  // Stage the tile: 16-byte chunks (NC = 4: half a point; NC = 1: two points).
  constexpr int kChunksPerRow = TX * NC / 2;
  for (int t = threadIdx.x; t < TZ * TY * kChunksPerRow; t += blockDim.x) {
    const int row = t / kChunksPerRow, h = t - row * kChunksPerRow;
    const int z = row / TY, y = row - z * TY;
    const int x = NC == 4 ? h / 2 : 2 * h;  // first point of the chunk
    double* dst = sG + row * RS + 2 * h;
    if (z < ez && y < ey && x < ex) {
      const R* src = grid + ((static_cast<size_t>(z0 + z) * sd.n[1] + y0 + y) * sd.n[0] + x0) * NC + 2 * h;
      stage2(dst, src);
    } else {
      dst[0] = 0.0;
      dst[1] = 0.0;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int fr = lane >> 2, fk = lane & 3;
  const int nslots = sd.pstride;
  for (int b0 = p0; b0 < p1; b0 += kGatherAtoms) {
    const int nb = min(kGatherAtoms, p1 - b0);
    __syncthreads();  // the previous round's weights are no longer read
    for (int a = threadIdx.x; a < kGatherAtoms; a += blockDim.x) {
      if (a < nb) {
        const int2 pr = pairs[b0 + a];
        sPair[a] = pr;
        const R* wk = wtab + static_cast<size_t>(pr.x) * sd.wstride;
        const R* src[3] = {wk + sd.woff[0] + (pr.y & 0xff) * TX,
                           wk + sd.woff[1] + ((pr.y >> 8) & 0xff) * TY,
                           wk + sd.woff[2] + (pr.y >> 16) * TZ};
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
          for (int j = 0; j < 4; ++j) stage2(&sW[d][a][2 * j], src[d] + 2 * j);
      } else {  // rows past the list: zero weights, results discarded
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
          for (int j = 0; j < 8; ++j) sW[d][a][j] = 0.0;
      }
    }
    cp_async_wait_all();  // also completes the tile copies on the first round
    __syncthreads();
    // This warp's M blocks: atoms warp * 32 + mb * 8 + (0..7) of the round.
    const int abase = warp * (MB * 8);
    if (abase >= nb) continue;
    const int nmb = min(MB, (nb - abase + 7) / 8);
    double fa[MB][2], cacc[MB][NC][2];
#pragma unroll
    for (int mb = 0; mb < MB; ++mb) {
      const int am = abase + mb * 8 + fr;  // this lane's atom row
      fa[mb][0] = sW[0][am][fk];           // A[m][k], k-step 0: x = k
      fa[mb][1] = sW[0][am][4 + fk];       // k-step 1: x = 4 + k
#pragma unroll
      for (int c = 0; c < NC; ++c) cacc[mb][c][0] = cacc[mb][c][1] = 0.0;
    }
    // w3 is folded into the A fragment, so C sums over z as well:
    // C[m][y] = sum_z sum_x w3_m(z) w1_m(x) G[z][y][x][c].
#pragma unroll 1
    for (int z = 0; z < TZ; ++z) {
      double a0[MB], a1[MB];
#pragma unroll
      for (int mb = 0; mb < MB; ++mb) {
        const double w3 = sW[2][abase + mb * 8 + fr][z];
        a0[mb] = fa[mb][0] * w3;
        a1[mb] = fa[mb][1] * w3;
      }
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        // B[k][n] = G[z][y = n][x = 4 ks + k][c] at lane 4n + k.
        const double* gz = sG + (z * TY + fr) * RS + c;
        const double b0v = gz[fk * NC];
        const double b1v = gz[(4 + fk) * NC];
#pragma unroll
        for (int mb = 0; mb < MB; ++mb) {
          if (mb < nmb) {
            dmma_m8n8k4(cacc[mb][c][0], cacc[mb][c][1], a0[mb], b0v);
            dmma_m8n8k4(cacc[mb][c][0], cacc[mb][c][1], a1[mb], b1v);
          }
        }
      }
    }
#pragma unroll
    for (int mb = 0; mb < MB; ++mb) {
      if (mb >= nmb) break;
      // This lane holds C for y = 2 fk and 2 fk + 1: weight them by w2 and sum
      // the four lanes of the atom.
      const int am = abase + mb * 8 + fr;
      const double w20 = sW[1][am][2 * fk], w21 = sW[1][am][2 * fk + 1];
      double acc[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        acc[c] = fma(w20, cacc[mb][c][0], w21 * cacc[mb][c][1]);
        acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 1);
        acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 2);
      }
      const int a = abase + mb * 8 + fr;
      if (fk == 0 && a < nb) {
        const int2 pr = sPair[a];
        const int ps = pr.y;
        const int sidx = ((ps >> 16) * sd.S[1] + ((ps >> 8) & 0xff)) * sd.S[0] + (ps & 0xff);
        double* dst = part + (static_cast<size_t>(pr.x) * nslots + sidx) * NC;
#pragma unroll
        for (int c = 0; c < NC; ++c) dst[c] = acc[c];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// FP64 gather with window derivatives (force scheme ad) on the tensor cores.
// The tile holds the potential grid alone.  Per plane z the x contraction
// takes two A operands that do not change from plane to plane, w1 and dw1:
//   C_w[z][m][y] = sum_x w1_m(x) G[z][y][x],  C_d[z][m][y] = sum_x dw1_m(x) G[z][y][x]
// (four DMMAs per plane for 8 atoms, each plane its own accumulators, so the
// 32 DMMAs of a tile are independent), and the y and z weights are applied
// afterwards:
//   phi = sum_z w3 sum_y w2 C_w,  D_1 = sum_z w3 sum_y w2 C_d,
//   D_2 = sum_z w3 sum_y dw2 C_w,  D_3 = sum_z dw3 sum_y w2 C_w.
// WARPS warps per tile, each taking blocks of 8 atoms (one M block) on its own.
// Shared layout and fragment mapping as in k_gather_tiles_dmma with NC = 1; six
// weight rows per atom (w1 w2 w3 dw1 dw2 dw3).
// ---------------------------------------------------------------------------
template <typename R, int WARPS>
__device__ __forceinline__ void gather_tiles_dmma_ad_body(
    int tx, int ty, int tz, const int* __restrict__ tile_start, const int2* __restrict__ pairs,
    const R* __restrict__ wtab, StencilDims sd, const R* __restrict__ grid,
    double* __restrict__ part) {
  chain_enter();
  constexpr int RS = GatherRow<1>::value;
  __shared__ __align__(16) double sG[TZ * TY * RS];
  __shared__ __align__(16) double sW[WARPS][6][8][kWRow];  // per warp: its 8 atoms' rows
  const int tile = (tz * sd.ntiles[1] + ty) * sd.ntiles[0] + tx;
  const int p0 = tile_start[tile], p1 = tile_start[tile + 1];
  if (p0 == p1) return;  // no atom reaches this tile
  const int x0 = tx * TX, y0 = ty * TY, z0 = tz * TZ;
  const int ex = min(TX, sd.n[0] - x0), ey = min(TY, sd.n[1] - y0), ez = min(TZ, sd.n[2] - z0);
  // Stage the tile: 16-byte chunks of two points.
  constexpr int kChunksPerRow = TX / 2;
  for (int t = threadIdx.x; t < TZ * TY * kChunksPerRow; t += blockDim.x) {
    const int row = t / kChunksPerRow, h = t - row * kChunksPerRow;
    const int z = row / TY, y = row - z * TY;
    const int x = 2 * h;
    double* dst = sG + row * RS + 2 * h;
    if (z < ez && y < ey && x < ex) {
      stage2(dst, grid + (static_cast<size_t>(z0 + z) * sd.n[1] + y0 + y) * sd.n[0] + x0 + x);
    } else {
      dst[0] = 0.0;
      dst[1] = 0.0;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int fr = lane >> 2, fk = lane & 3;
  const int nslots = sd.pstride;
  double(*W)[8][kWRow] = sW[warp];
  cp_async_wait_all();
  __syncthreads();  // the tile, staged by all warps; the only CTA barrier
  // Each warp takes blocks of 8 atoms of the tile's list on its own.  Lane
  // (fr, fk) stages 16-byte chunk fk of atom fr's six rows and later holds
  // that atom's fragments.
  for (int b0 = p0 + warp * 8; b0 < p1; b0 += WARPS * 8) {
    const int nb = min(8, p1 - b0);
    __syncwarp();  // the previous block's rows are no longer read
    int2 pr = make_int2(0, 0);
    if (fr < nb) {
      pr = pairs[b0 + fr];
      const R* wk = wtab + static_cast<size_t>(pr.x) * sd.wstride;
      const int off[3] = {sd.woff[0] + (pr.y & 0xff) * TX, sd.woff[1] + ((pr.y >> 8) & 0xff) * TY,
                          sd.woff[2] + (pr.y >> 16) * TZ};
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        stage2(&W[d][fr][2 * fk], wk + off[d] + 2 * fk);
        stage2(&W[3 + d][fr][2 * fk], wk + sd.dwoff + off[d] + 2 * fk);
      }
    } else {  // rows past the list: zero weights, results discarded
#pragma unroll
      for (int d = 0; d < 6; ++d) W[d][fr][2 * fk] = W[d][fr][2 * fk + 1] = 0.0;
    }
    cp_async_wait_all();
    __syncwarp();
    const double fw0 = W[0][fr][fk], fw1 = W[0][fr][4 + fk];
    const double fd0 = W[3][fr][fk], fd1 = W[3][fr][4 + fk];
    double cw[TZ][2], cd[TZ][2];
#pragma unroll
    for (int z = 0; z < TZ; ++z) {
      // B[k][n] = G[z][y = n][x = 4 ks + k] at lane 4n + k.
      const double* gz = sG + (z * TY + fr) * RS;
      const double b0v = gz[fk], b1v = gz[4 + fk];
      cw[z][0] = cw[z][1] = cd[z][0] = cd[z][1] = 0.0;
      dmma_m8n8k4(cw[z][0], cw[z][1], fw0, b0v);
      dmma_m8n8k4(cw[z][0], cw[z][1], fw1, b1v);
      dmma_m8n8k4(cd[z][0], cd[z][1], fd0, b0v);
      dmma_m8n8k4(cd[z][0], cd[z][1], fd1, b1v);
    }
    // This lane holds C for y = 2 fk and 2 fk + 1 of every plane.
    const double w20 = W[1][fr][2 * fk], w21 = W[1][fr][2 * fk + 1];
    const double d20 = W[4][fr][2 * fk], d21 = W[4][fr][2 * fk + 1];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int z = 0; z < TZ; ++z) {
      const double w3 = W[2][fr][z], d3 = W[5][fr][z];
      const double pw = fma(w20, cw[z][0], w21 * cw[z][1]);
      const double pd = fma(w20, cd[z][0], w21 * cd[z][1]);
      const double qw = fma(d20, cw[z][0], d21 * cw[z][1]);
      acc[0] = fma(w3, pw, acc[0]);
      acc[1] = fma(w3, pd, acc[1]);
      acc[2] = fma(w3, qw, acc[2]);
      acc[3] = fma(d3, pw, acc[3]);
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 1);
      acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 2);
    }
    if (fk == 0 && fr < nb) {
      const int ps = pr.y;
      const int sidx = ((ps >> 16) * sd.S[1] + ((ps >> 8) & 0xff)) * sd.S[0] + (ps & 0xff);
      double* dst = part + (static_cast<size_t>(pr.x) * nslots + sidx) * 4;
#pragma unroll
      for (int c = 0; c < 4; ++c) dst[c] = acc[c];
    }
  }
}

// Final per-atom sum of the slot partials in a fixed order, with the assembly
// of fft/ewald_fft_3d.f90:121-132: pot = (sr + lr) + self, force = sr + q lr.
// A group of lanes per atom (a warp, or 8 lanes when the atom has at most 32
// slots) reads the atom's slots (contiguous, coalesced), then a shuffle tree
// sums them (a fixed order: results are reproducible).
// Dual basis rows for the ad partials (on = 0: ik partials, Cartesian already).
struct RecRows {
  double b[3][3];
  int on;
};

// LPA lanes per atom (32, or 8 when an atom has at most 32 slots: four atoms
// per warp).
template <int NC, int LPA>
__device__ __forceinline__ void gather_final_body(const int4* __restrict__ slot,
                                                  const int* __restrict__ perm,
                                                  const double* __restrict__ part, int k,
                                                  int lane, bool live, const StencilDims& sd,
                                                  const double* __restrict__ q, double self_coef,
                                                  double pot_shift,
                                                  const double* __restrict__ pot_sr,
                                                  const double* __restrict__ f_sr,
                                                  double* __restrict__ pot,
                                                  double* __restrict__ force, const RecRows& rr) {
  const int4 si = live ? slot[k] : make_int4(0, 0, 0, 0);
  const int cx = slot_count(si.x), cy = slot_count(si.y), cz = slot_count(si.z);
  const int nslots = sd.S[0] * sd.S[1] * sd.S[2];
  const double* pk = part + static_cast<size_t>(live ? k : 0) * sd.pstride * NC;
  double acc[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) acc[c] = 0.0;
  for (int s = lane; s < (live ? nslots : 0); s += LPA) {
    const int sx = s % sd.S[0], sy = (s / sd.S[0]) % sd.S[1], sz = s / (sd.S[0] * sd.S[1]);
    if (sx < cx && sy < cy && sz < cz) {  // slots past the atom's tiles hold no partial
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[c] += pk[s * NC + c];
    }
  }
  // A fixed shuffle tree within the atom's LPA lanes.
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int off = LPA / 2; off > 0; off >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], off);
  if (lane != 0 || !live) return;
  const int i = perm[k];
  const double qi = q[i];
  pot[i] = (pot_sr[i] + acc[0]) + self_coef * qi + pot_shift;
  if (NC == 4 && force) {
    if (rr.on) {  // ad: F = -q sum_e D_e b_e, D_e the derivative along s_e
#pragma unroll
      for (int d = 0; d < 3; ++d)
        force[3 * i + d] =
            f_sr[3 * i + d] - qi * (acc[1] * rr.b[0][d] + acc[2] * rr.b[1][d] + acc[3] * rr.b[2][d]);
    } else {
#pragma unroll
      for (int d = 0; d < 3; ++d) force[3 * i + d] = f_sr[3 * i + d] + qi * acc[1 + d];
    }
  }
}

template <int NC, int LPA>
__global__ void k_gather_final(const int4* __restrict__ slot, const int* __restrict__ perm,
                               const double* __restrict__ part, int n, StencilDims sd,
                               const double* __restrict__ q, double self_coef, double pot_shift,
                               const double* __restrict__ pot_sr, const double* __restrict__ f_sr,
                               double* __restrict__ pot, double* __restrict__ force, RecRows rr) {
  const long t = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int k = static_cast<int>(t / LPA);
  // Lanes past the last atom stay to the end: the shuffles below take the whole warp.
  gather_final_body<NC, LPA>(slot, perm, part, k, static_cast<int>(t % LPA), k < n, sd, q,
                             self_coef, pot_shift, pot_sr, f_sr, pot, force, rr);
}

// Every cell of a batch: the atom's cell gives its slot layout, self term and
// dual basis (window-derivative partials are fractional derivatives).
template <int NC, int LPA>
__global__ void k_gather_final_seg(const BatchCell* __restrict__ cells,
                                   const int* __restrict__ prefix, int ncells,
                                   const int4* __restrict__ slot, const int* __restrict__ perm,
                                   const double* __restrict__ part, int n,
                                   const double* __restrict__ q, const double* __restrict__ pot_sr,
                                   const double* __restrict__ f_sr, double* __restrict__ pot,
                                   double* __restrict__ force) {
  const long t = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int k = static_cast<int>(t / LPA);
  const bool live = k < n;
  const BatchCell& bc = cells[seg_cell(prefix, ncells, live ? k : n - 1)];
  RecRows rr;
  rr.on = 1;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int d = 0; d < 3; ++d) rr.b[a][d] = bc.rec[a][d];
  const StencilDims sd = bc.sd;
  gather_final_body<NC, LPA>(slot, perm, part, k, static_cast<int>(t % LPA), live, sd, q,
                             bc.self_coef, 0.0, pot_sr, f_sr, pot, force, rr);
}

// FP64 tensor-core throughput probe: every warp issues independent DMMAs on
// register operands (eight accumulator pairs, no memory traffic), so the
// measured rate is the m8n8k4 FP64 pipe's own.
__global__ void __launch_bounds__(128) k_dmma_peak(int iters, double seed, double* sink) {
  double acc[8][2];
#pragma unroll
  for (int i = 0; i < 8; ++i) acc[i][0] = acc[i][1] = 0.0;
  const double a = seed + 1.0e-9 * threadIdx.x, b = 1.0 - seed;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) dmma_m8n8k4(acc[i][0], acc[i][1], a, b);
  }
  double t = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) t += acc[i][0] + acc[i][1];
  if (t == -1.0) sink[threadIdx.x] = t;  // never true; keeps the work live
}

// ---- the tile kernels: one tile per CTA (blockIdx = tile), or, for a batch,
// the tiles of every cell (blockIdx.x over the cells' tiles end to end; the
// cell's tile list, weights layout and grid from the batch table).
__device__ __forceinline__ const BatchCell& tile_of_block(const BatchCell* __restrict__ cells,
                                                          const int* __restrict__ prefix,
                                                          int ncells, int* tx, int* ty, int* tz) {
  const int c = seg_cell(prefix, ncells, blockIdx.x);
  const BatchCell& bc = cells[c];
  const int local = static_cast<int>(blockIdx.x) - prefix[c];
  *tx = local % bc.sd.ntiles[0];
  *ty = (local / bc.sd.ntiles[0]) % bc.sd.ntiles[1];
  *tz = local / (bc.sd.ntiles[0] * bc.sd.ntiles[1]);
  return bc;
}

template <typename R>
__global__ void __launch_bounds__(kSpreadLanes) k_spread_tiles(const int* __restrict__ tile_start,
                                                               const int2* __restrict__ pairs,
                                                               const R* __restrict__ wtab,
                                                               const R* __restrict__ qk,
                                                               StencilDims sd, R* __restrict__ grid) {
  spread_tiles_body<R>(blockIdx.x, blockIdx.y, blockIdx.z, tile_start, pairs, wtab, qk, sd, grid);
}
template <typename R>
__global__ void __launch_bounds__(32) k_spread_tiles_dmma(const int* __restrict__ tile_start,
                                                          const int2* __restrict__ pairs,
                                                          const R* __restrict__ wtab,
                                                          const R* __restrict__ qk,
                                                          StencilDims sd, R* __restrict__ grid) {
  spread_tiles_dmma_body<R>(blockIdx.x, blockIdx.y, blockIdx.z, tile_start, pairs, wtab, qk, sd,
                            grid);
}
template <typename R>
__global__ void __launch_bounds__(32) k_spread_tiles_dmma_seg(
    const BatchCell* __restrict__ cells, const int* __restrict__ prefix, int ncells,
    const int* __restrict__ tile_start, const int2* __restrict__ pairs,
    const R* __restrict__ wtab, const R* __restrict__ qk) {
  int tx, ty, tz;
  const BatchCell& bc = tile_of_block(cells, prefix, ncells, &tx, &ty, &tz);
  spread_tiles_dmma_body<R>(tx, ty, tz, tile_start + bc.tile0, pairs, wtab, qk, bc.sd,
                            static_cast<R*>(bc.grid));
}

template <typename R, int NC, int A, int WARPS>
__global__ void __launch_bounds__(32 * WARPS) k_gather_tiles(const int* __restrict__ tile_start,
                                                             const int2* __restrict__ pairs,
                                                             const R* __restrict__ wtab,
                                                             StencilDims sd,
                                                             const R* __restrict__ grid,
                                                             double* __restrict__ part) {
  gather_tiles_body<R, NC, A, WARPS>(blockIdx.x, blockIdx.y, blockIdx.z, tile_start, pairs, wtab,
                                     sd, grid, part);
}
template <int A, int WARPS>
__global__ void __launch_bounds__(32 * WARPS) k_gather_tiles_ad(const int* __restrict__ tile_start,
                                                                const int2* __restrict__ pairs,
                                                                const float* __restrict__ wtab,
                                                                StencilDims sd,
                                                                const float* __restrict__ grid,
                                                                double* __restrict__ part) {
  gather_tiles_ad_body<A, WARPS>(blockIdx.x, blockIdx.y, blockIdx.z, tile_start, pairs, wtab, sd,
                                 grid, part);
}
template <typename R, int NC, int WARPS, int MB>
__global__ void __launch_bounds__(32 * WARPS) k_gather_tiles_dmma(const int* __restrict__ tile_start,
                                                                  const int2* __restrict__ pairs,
                                                                  const R* __restrict__ wtab,
                                                                  StencilDims sd,
                                                                  const R* __restrict__ grid,
                                                                  double* __restrict__ part) {
  gather_tiles_dmma_body<R, NC, WARPS, MB>(blockIdx.x, blockIdx.y, blockIdx.z, tile_start, pairs,
                                           wtab, sd, grid, part);
}
template <typename R, int NC, int WARPS, int MB>
__global__ void __launch_bounds__(32 * WARPS) k_gather_tiles_dmma_seg(
    const BatchCell* __restrict__ cells, const int* __restrict__ prefix, int ncells,
    const int* __restrict__ tile_start, const int2* __restrict__ pairs,
    const R* __restrict__ wtab, double* __restrict__ part) {
  int tx, ty, tz;
  const BatchCell& bc = tile_of_block(cells, prefix, ncells, &tx, &ty, &tz);
  gather_tiles_dmma_body<R, NC, WARPS, MB>(tx, ty, tz, tile_start + bc.tile0, pairs, wtab, bc.sd,
                                           static_cast<const R*>(bc.out), part);
}

template <typename R, int WARPS>
__global__ void __launch_bounds__(32 * WARPS) k_gather_tiles_dmma_ad(
    const int* __restrict__ tile_start, const int2* __restrict__ pairs,
    const R* __restrict__ wtab, StencilDims sd, const R* __restrict__ grid,
    double* __restrict__ part) {
  gather_tiles_dmma_ad_body<R, WARPS>(blockIdx.x, blockIdx.y, blockIdx.z, tile_start, pairs, wtab,
                                      sd, grid, part);
}
template <typename R, int WARPS>
__global__ void __launch_bounds__(32 * WARPS) k_gather_tiles_dmma_ad_seg(
    const BatchCell* __restrict__ cells, const int* __restrict__ prefix, int ncells,
    const int* __restrict__ tile_start, const int2* __restrict__ pairs,
    const R* __restrict__ wtab, double* __restrict__ part) {
  int tx, ty, tz;
  const BatchCell& bc = tile_of_block(cells, prefix, ncells, &tx, &ty, &tz);
  gather_tiles_dmma_ad_body<R, WARPS>(tx, ty, tz, tile_start + bc.tile0, pairs, wtab, bc.sd,
                                      static_cast<const R*>(bc.out), part);
}

template <typename R>
__global__ void k_sorted_charges(const double* __restrict__ q, const int* __restrict__ perm, int n,
                                 R* __restrict__ qk) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) qk[k] = static_cast<R>(q[perm[k]]);
}

inline int blocks_for(long n, int threads) { return static_cast<int>((n + threads - 1) / threads); }

}  // namespace

void launch_weights(const MeshPlan& mp, const int4* mc, const double4* fr, const int* perm, int n,
                    void* wtab, void* qk, int4* slot, cudaStream_t st) {
  if (n == 0) return;
  const long threads = static_cast<long>(mp.sd.S[0] + mp.sd.S[1] + mp.sd.S[2]) * n;
  if (mp.mixed)
    launch_chained(k_weights_tiled<float>, blocks_for(threads, 128), 128, 0, st,
        mc, fr, perm, n, mp.sd, static_cast<float*>(wtab), static_cast<float*>(qk), slot);
  else
    launch_chained(k_weights_tiled<double>, blocks_for(threads, 128), 128, 0, st,
        mc, fr, perm, n, mp.sd, static_cast<double*>(wtab), static_cast<double*>(qk), slot);
  ++g_launches;
}

void launch_sorted_charges(const MeshPlan& mp, const double* q, const int* perm, int n, void* qk,
                           cudaStream_t st) {
  if (n == 0) return;
  if (mp.mixed)
    k_sorted_charges<float><<<blocks_for(n, 256), 256, 0, st>>>(q, perm, n, static_cast<float*>(qk));
  else
    k_sorted_charges<double><<<blocks_for(n, 256), 256, 0, st>>>(q, perm, n, static_cast<double*>(qk));
  ++g_launches;
}

void launch_pair_bins(const MeshPlan& mp, const int4* slot, int n, int* counts, int* cursor,
                      int* tile_start, int4* tmp, int2* pairs, int npairs_max, cudaStream_t st) {
  const int ntiles = mp.sd.ntiles[0] * mp.sd.ntiles[1] * mp.sd.ntiles[2];
  const long nthreads = static_cast<long>(n) * mp.sd.S[0] * mp.sd.S[1] * mp.sd.S[2];
  int2* t2 = reinterpret_cast<int2*>(tmp);
  cudaMemsetAsync(counts, 0, sizeof(int) * ntiles, st);
  cudaMemsetAsync(cursor, 0, sizeof(int) * ntiles, st);
  if (n > 0) {
    k_pair_count<<<blocks_for(nthreads, 256), 256, 0, st>>>(slot, n, mp.sd, counts);
    ++g_launches;
  }
  launch_scan(counts, ntiles, tile_start, n > 0, st);
  if (n > 0) {
    launch_chained(k_pair_scatter, blocks_for(nthreads, 256), 256, 0, st, slot, n, mp.sd, tile_start, cursor,
                                                               t2);
    launch_chained(k_pair_rank, blocks_for(npairs_max, 256), 256, 0, st, t2, tile_start, ntiles, slot, mp.sd,
                                                              pairs);
    g_launches += 2;
  }
}

void launch_spread(const MeshPlan& mp, const int* tile_start, const int2* pairs, const void* wtab,
                   const void* qk, void* grid, cudaStream_t st) {
  dim3 grd(mp.sd.ntiles[0], mp.sd.ntiles[1], mp.sd.ntiles[2]);
  if (mp.mixed && mp.stencil == 2)  // FP32 CUDA-core spread
    launch_chained(k_spread_tiles<float>, grd, kSpreadLanes, 0, st, tile_start, pairs,
                   static_cast<const float*>(wtab), static_cast<const float*>(qk), mp.sd,
                   static_cast<float*>(grid));
  else if (mp.mixed)  // FP32 weights and grid, FP64 products on the tensor cores
    launch_chained(k_spread_tiles_dmma<float>, grd, 32, 0, st, tile_start, pairs,
                   static_cast<const float*>(wtab), static_cast<const float*>(qk), mp.sd,
                   static_cast<float*>(grid));
  else
    launch_chained(k_spread_tiles_dmma<double>, grd, 32, 0, st, tile_start, pairs,
                   static_cast<const double*>(wtab), static_cast<const double*>(qk), mp.sd,
                   static_cast<double*>(grid));
  ++g_launches;
}

void launch_gather(const MeshPlan& mp, const int* tile_start, const int2* pairs, const void* wtab,
                   const void* grid, int nc, double* part, cudaStream_t st) {
  dim3 grd(mp.sd.ntiles[0], mp.sd.ntiles[1], mp.sd.ntiles[2]);
#define EWG_GATHER(R, NC)                                                                \
  launch_chained(k_gather_tiles<R, NC, GatherShape<R>::atoms, GatherShape<R>::warps>, grd,  \
                 32 * GatherShape<R>::warps, 0, st, tile_start, pairs,                       \
                 static_cast<const R*>(wtab), mp.sd, static_cast<const R*>(grid), part)
  const bool cores = mp.mixed && mp.stencil == 2;  // FP32 CUDA-core stencils
  if (mp.sd.ad && nc == 1) {  // force wanted, ad scheme: potential grid, four partials
    if (cores)
      launch_chained(k_gather_tiles_ad<kGatherAdF32Atoms, kGatherAdF32Warps>, grd,
                     32 * kGatherAdF32Warps, 0, st, tile_start, pairs,
                     static_cast<const float*>(wtab), mp.sd, static_cast<const float*>(grid), part);
    else if (mp.mixed)
      launch_chained(k_gather_tiles_dmma_ad<float, kGatherAdWarps>, grd, 32 * kGatherAdWarps, 0,
                     st, tile_start, pairs, static_cast<const float*>(wtab), mp.sd,
                     static_cast<const float*>(grid), part);
    else
      launch_chained(k_gather_tiles_dmma_ad<double, kGatherAdWarps>, grd, 32 * kGatherAdWarps, 0,
                     st, tile_start, pairs, static_cast<const double*>(wtab), mp.sd,
                     static_cast<const double*>(grid), part);
  } else if (cores) {
    if (nc == 4)
      EWG_GATHER(float, 4);
    else
      EWG_GATHER(float, 1);
  } else {
    // The kernel shape's warps per tile; every shape stages 64 atoms per round
    // (warps x blocks of 8 atoms per warp) and gives bitwise the same partials.
#define EWG_GATHER64(R, NC, WARPS, MB)                                                          \
  launch_chained(k_gather_tiles_dmma<R, NC, WARPS, MB>, grd, 32 * WARPS, 0, st, tile_start, pairs, \
                 static_cast<const R*>(wtab), mp.sd, static_cast<const R*>(grid), part)
#define EWG_GATHER64_SHAPES(R, NC)          \
  do {                                      \
    if (mp.gather_warps == 2)               \
      EWG_GATHER64(R, NC, 2, 4);            \
    else if (mp.gather_warps == 8)          \
      EWG_GATHER64(R, NC, 8, 1);            \
    else                                    \
      EWG_GATHER64(R, NC, kGatherWarps, kGatherMB); \
  } while (0)
    static_assert(kGatherWarps * kGatherMB == 8, "64 atoms per round");
    if (mp.mixed) {  // FP32 tiles and weights, FP64 products on the tensor cores
      if (nc == 4)
        EWG_GATHER64_SHAPES(float, 4);
      else
        EWG_GATHER64_SHAPES(float, 1);
    } else {
      if (nc == 4)
        EWG_GATHER64_SHAPES(double, 4);
      else
        EWG_GATHER64_SHAPES(double, 1);
    }
#undef EWG_GATHER64_SHAPES
#undef EWG_GATHER64
  }
#undef EWG_GATHER
  ++g_launches;
}

void launch_gather_final(const MeshPlan& mp, const int4* slot, const int* perm, const double* part,
                         int nparts, int n, const double* q, double self_coef, double pot_shift,
                         const double* pot_sr, const double* f_sr, double* pot, double* force,
                         const double (*rec)[3], cudaStream_t st) {
  if (n == 0) return;
  RecRows rr{};
  if (rec) {
    rr.on = 1;
    for (int i = 0; i < 3; ++i)
      for (int d = 0; d < 3; ++d) rr.b[i][d] = rec[i][d];
  }
  const bool narrow = mp.sd.S[0] * mp.sd.S[1] * mp.sd.S[2] <= 32;
  if (nparts == 4) {
    if (narrow)
      k_gather_final<4, 8><<<blocks_for(8L * n, 256), 256, 0, st>>>(
          slot, perm, part, n, mp.sd, q, self_coef, pot_shift, pot_sr, f_sr, pot, force, rr);
    else
      k_gather_final<4, 32><<<blocks_for(32L * n, 256), 256, 0, st>>>(
          slot, perm, part, n, mp.sd, q, self_coef, pot_shift, pot_sr, f_sr, pot, force, rr);
  } else {
    if (narrow)
      k_gather_final<1, 8><<<blocks_for(8L * n, 256), 256, 0, st>>>(
          slot, perm, part, n, mp.sd, q, self_coef, pot_shift, pot_sr, f_sr, pot, nullptr, rr);
    else
      k_gather_final<1, 32><<<blocks_for(32L * n, 256), 256, 0, st>>>(
          slot, perm, part, n, mp.sd, q, self_coef, pot_shift, pot_sr, f_sr, pot, nullptr, rr);
  }
  ++g_launches;
}

void launch_weights_seg(const BatchLaunch& b, const int4* mc, const double4* fr, const int* perm,
                        void* wtab, void* qk, int4* slot, cudaStream_t st) {
  if (b.n_weights == 0) return;
  if (b.mixed)
    launch_chained(k_weights_seg<float>, blocks_for(b.n_weights, 128), 128, 0, st, b.cells,
                   b.p_weights, b.ncells, b.n_weights, mc, fr, perm, static_cast<float*>(wtab),
                   static_cast<float*>(qk), slot);
  else
    launch_chained(k_weights_seg<double>, blocks_for(b.n_weights, 128), 128, 0, st, b.cells,
                   b.p_weights, b.ncells, b.n_weights, mc, fr, perm, static_cast<double*>(wtab),
                   static_cast<double*>(qk), slot);
  ++g_launches;
}

void launch_pair_bins_seg(const BatchLaunch& b, const int4* slot, int* counts, int* cursor,
                          int* tile_start, int4* tmp, int2* pairs, cudaStream_t st) {
  int2* t2 = reinterpret_cast<int2*>(tmp);
  cudaMemsetAsync(counts, 0, sizeof(int) * b.n_tiles, st);
  cudaMemsetAsync(cursor, 0, sizeof(int) * b.n_tiles, st);
  if (b.n_slots > 0) {
    k_pair_count_seg<<<blocks_for(b.n_slots, 256), 256, 0, st>>>(b.cells, b.p_slots, b.ncells,
                                                                 b.n_slots, slot, counts);
    ++g_launches;
  }
  launch_scan(counts, b.n_tiles, tile_start, b.n_slots > 0, st);
  if (b.n_slots > 0) {
    launch_chained(k_pair_scatter_seg, blocks_for(b.n_slots, 256), 256, 0, st, b.cells, b.p_slots,
                   b.ncells, b.n_slots, slot, tile_start, cursor, t2);
    launch_chained(k_pair_rank_seg, blocks_for(b.n_slots, 256), 256, 0, st, b.cells, b.p_atoms,
                   b.ncells, t2, tile_start, b.n_tiles, slot, pairs);
    g_launches += 2;
  }
}

void launch_spread_seg(const BatchLaunch& b, const int* tile_start, const int2* pairs,
                       const void* wtab, const void* qk, cudaStream_t st) {
  if (b.n_tiles == 0) return;
  if (b.mixed)
    launch_chained(k_spread_tiles_dmma_seg<float>, b.n_tiles, 32, 0, st, b.cells, b.p_tiles,
                   b.ncells, tile_start, pairs, static_cast<const float*>(wtab),
                   static_cast<const float*>(qk));
  else
    launch_chained(k_spread_tiles_dmma_seg<double>, b.n_tiles, 32, 0, st, b.cells, b.p_tiles,
                   b.ncells, tile_start, pairs, static_cast<const double*>(wtab),
                   static_cast<const double*>(qk));
  ++g_launches;
}

void launch_gather_seg(const BatchLaunch& b, const int* tile_start, const int2* pairs,
                       const void* wtab, double* part, cudaStream_t st) {
  if (b.n_tiles == 0) return;
  const int nb = b.n_tiles;
  if (b.ad && b.nc == 1 && b.nparts == 4) {  // window-differentiated forces
    if (b.mixed)
      launch_chained(k_gather_tiles_dmma_ad_seg<float, kGatherAdWarps>, nb, 32 * kGatherAdWarps, 0,
                     st, b.cells, b.p_tiles, b.ncells, tile_start, pairs,
                     static_cast<const float*>(wtab), part);
    else
      launch_chained(k_gather_tiles_dmma_ad_seg<double, kGatherAdWarps>, nb, 32 * kGatherAdWarps,
                     0, st, b.cells, b.p_tiles, b.ncells, tile_start, pairs,
                     static_cast<const double*>(wtab), part);
  } else if (b.mixed) {
    const float* w = static_cast<const float*>(wtab);
    if (b.nc == 4)
      launch_chained(k_gather_tiles_dmma_seg<float, 4, kGatherWarps, kGatherMB>, nb,
                     32 * kGatherWarps, 0, st, b.cells, b.p_tiles, b.ncells, tile_start, pairs, w,
                     part);
    else
      launch_chained(k_gather_tiles_dmma_seg<float, 1, kGatherWarps, kGatherMB>, nb,
                     32 * kGatherWarps, 0, st, b.cells, b.p_tiles, b.ncells, tile_start, pairs, w,
                     part);
  } else {
    const double* w = static_cast<const double*>(wtab);
    if (b.nc == 4)
      launch_chained(k_gather_tiles_dmma_seg<double, 4, kGatherWarps, kGatherMB>, nb,
                     32 * kGatherWarps, 0, st, b.cells, b.p_tiles, b.ncells, tile_start, pairs, w,
                     part);
    else
      launch_chained(k_gather_tiles_dmma_seg<double, 1, kGatherWarps, kGatherMB>, nb,
                     32 * kGatherWarps, 0, st, b.cells, b.p_tiles, b.ncells, tile_start, pairs, w,
                     part);
  }
  ++g_launches;
}

void launch_gather_final_seg(const BatchLaunch& b, const int4* slot, const int* perm,
                             const double* part, const double* q, const double* pot_sr,
                             const double* f_sr, double* pot, double* force, cudaStream_t st) {
  if (b.n_atoms == 0) return;
  const int n = b.n_atoms;
  const int blocks = blocks_for(static_cast<long>(b.lpa) * n, 256);
#define EWG_FINAL(NC, LPA)                                                                   \
  k_gather_final_seg<NC, LPA><<<blocks, 256, 0, st>>>(b.cells, b.p_atoms, b.ncells, slot, perm, \
                                                      part, n, q, pot_sr, f_sr, pot,         \
                                                      NC == 4 ? force : nullptr)
  if (b.nparts == 4) {
    if (b.lpa == 8)
      EWG_FINAL(4, 8);
    else
      EWG_FINAL(4, 32);
  } else {
    if (b.lpa == 8)
      EWG_FINAL(1, 8);
    else
      EWG_FINAL(1, 32);
  }
#undef EWG_FINAL
  ++g_launches;
}

int stencil_configure_kernels() { return EWG_OK; }

int measure_dmma_peak(cudaStream_t st, double* tflops) {
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return EWG_ERR_CUDA;
  const int blocks = 4 * nsm, threads = 128, iters = 4096;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return EWG_ERR_CUDA;
  k_dmma_peak<<<blocks, threads, 0, st>>>(iters / 8, 0.25, nullptr);  // warm-up
  cudaEventRecord(e0, st);
  k_dmma_peak<<<blocks, threads, 0, st>>>(iters, 0.25, nullptr);
  cudaEventRecord(e1, st);
  g_launches += 2;
  float ms = 0.0f;
  const bool ok = cudaEventSynchronize(e1) == cudaSuccess &&
                  cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && ms > 0.0f;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!ok) return EWG_ERR_CUDA;
  const double mmas = static_cast<double>(blocks) * (threads / 32) * iters * 8;
  *tflops = mmas * 2.0 * 8 * 8 * 4 / (ms * 1e-3) / 1e12;
  return EWG_OK;
}

}  // namespace ewg
