// ewg_real.cu -- per-atom preparation, the deterministic bucket sort, the
// real-space erfc pair sum over a linked-cell layout, and the stock stress
// terms (real-space virial and reciprocal structure-factor sum).
//
// Cell list.  Boxes are at least r_cut wide along every dual direction
// (box_counts_3d, common/ewald_cell_list.f90:56-73).  An atom in box b meets
// every partner within r_cut among the boxes b - R .. b + R per axis, where
// R = ceil(r_cut |b_d| nb_d); R = 1 whenever at least one box fits, so the
// usual case is the reference's 27-box neighbourhood (fft/ewald_fft_3d_real.f90:143-180),
// and a cell narrower than the cutoff enumerates periodic images the way the
// direct engine's explicit image sum does (direct/ewald_direct_3d.f90:236-298).
// Boxes adjacent along x are contiguous in the sorted order, so each (dy, dz)
// row of neighbour boxes is scanned as at most a few contiguous runs.

#include <cuda_runtime.h>

#include <cmath>
#include <type_traits>

#include "ewg_kernels.h"

namespace ewg {

thread_local long long g_launches = 0;

namespace {

constexpr double kSqrtPi = 1.77245385090551602730;  // sqrt(pi)

// floor(a / n) for n > 0.  Box indices of a neighbourhood lie within one
// image of the cell almost always, which needs no division.
__device__ __forceinline__ int floor_div(int a, int n) {
  if (a >= 0 && a < n) return 0;
  if (a < 0 && a >= -n) return -1;
  if (a >= n && a < 2 * n) return 1;
  return a >= 0 ? a / n : -((-a + n - 1) / n);
}

// ---------------------------------------------------------------------------
// Atom preparation.  Fractional coordinates t = b_d . x (fft/ewald_fft_3d_fourier.f90:76-81),
// wrapped s = t - floor(t) (common/ewald_cell_list.f90:130-136), the box index
// min(int(s nb), nb - 1) (:78-91), and the mesh stencil origin: lowest grid
// point floor(s n) and the fraction s n - lowest (nfft/nfft.f90:148-152).
// ---------------------------------------------------------------------------
struct PrepArgs {
  double rec[3][3];
  int nb[3];
  int ng[3];
};

// One atom of k_atom_prep (key: its box in the cell's own numbering).
__device__ __forceinline__ void atom_prep_one(const double (&x)[3], double qi, const PrepArgs& a,
                                              int i, int key0, double4* __restrict__ s4,
                                              int* __restrict__ box_key,
                                              int4* __restrict__ mesh_c,
                                              double4* __restrict__ mesh_fr) {
  double s[3];
  int bx[3], c[3];
  double fr[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double t = a.rec[d][0] * x[0] + a.rec[d][1] * x[1] + a.rec[d][2] * x[2];
    s[d] = t - floor(t);
    if (a.nb[d] > 0) bx[d] = min(static_cast<int>(s[d] * a.nb[d]), a.nb[d] - 1);
    if (a.ng[d] > 0) {
      const double scaled = s[d] * a.ng[d];
      int lowest = static_cast<int>(floor(scaled));
      fr[d] = scaled - static_cast<double>(lowest);
      if (lowest >= a.ng[d]) lowest -= a.ng[d];
      c[d] = lowest;
    }
  }
  if (s4) s4[i] = make_double4(s[0], s[1], s[2], qi);
  if (box_key) box_key[i] = key0 + (bx[2] * a.nb[1] + bx[1]) * a.nb[0] + bx[0];
  if (mesh_c) {
    mesh_c[i] = make_int4(c[0], c[1], c[2], 0);
    mesh_fr[i] = make_double4(fr[0], fr[1], fr[2], qi);
  }
}

__global__ void k_atom_prep(const double* __restrict__ pos, long sa, long sd,
                            const double* __restrict__ q, int n, PrepArgs a,
                            double4* __restrict__ s4, int* __restrict__ box_key,
                            int4* __restrict__ mesh_c, double4* __restrict__ mesh_fr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x[3] = {pos[i * sa], pos[i * sa + sd], pos[i * sa + 2 * sd]};
  atom_prep_one(x, q[i], a, i, 0, s4, box_key, mesh_c, mesh_fr);
}

// Every cell of a batch at once: atom i of the global arrays (coords(3, total)),
// its cell's reciprocal rows, boxes and grid; box keys offset by the cell's box0.
__global__ void k_atom_prep_seg(const BatchCell* __restrict__ cells, const int* __restrict__ prefix,
                                int ncells, int n, const double* __restrict__ pos,
                                const double* __restrict__ q, double4* __restrict__ s4,
                                int* __restrict__ box_key, int4* __restrict__ mesh_c,
                                double4* __restrict__ mesh_fr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const BatchCell& bc = cells[seg_cell(prefix, ncells, i)];
  PrepArgs a;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
#pragma unroll
    for (int e = 0; e < 3; ++e) a.rec[d][e] = bc.rec[d][e];
    a.nb[d] = bc.rg.nb[d];
    a.ng[d] = bc.g.n[d];
  }
  const double x[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
  atom_prep_one(x, q[i], a, i, bc.box0, s4, box_key, mesh_c, mesh_fr);
}

// ---------------------------------------------------------------------------
// Bucket sort.  Counts and offsets are exact integers; the within-bucket order
// is made deterministic by ranking each atom among its bucket by index.
// ---------------------------------------------------------------------------
__global__ void k_count(const int* __restrict__ key, int n, int* __restrict__ counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(&counts[key[i]], 1);
}

// Exclusive scan of counts into starts[0..nkeys]; one CTA of 1024 threads.
// Each round stages 8192 counts in shared memory with coalesced loads, scans 8
// consecutive entries per thread and writes the starts back coalesced.  The
// next round's counts are loaded into registers while this round is scanned.
__global__ void __launch_bounds__(1024) k_scan(const int* __restrict__ counts, int nkeys,
                                               int* __restrict__ starts) {
  chain_enter();
  constexpr int kItems = 8, kRound = 1024 * kItems;
  __shared__ int buf[kRound + kRound / 32];  // padded: entry i at i + i / 32
  __shared__ int warp_sums[32];
  __shared__ int carry_s;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  int carry = 0;
  int next[kItems];
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    const int e = j * 1024 + tid;
    next[j] = e < nkeys ? counts[e] : 0;
  }
  for (int base = 0; base < nkeys; base += kRound) {
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      const int e = j * 1024 + tid;
      buf[e + (e >> 5)] = next[j];
    }
    if (base + kRound < nkeys) {
#pragma unroll
      for (int j = 0; j < kItems; ++j) {
        const int e = base + kRound + j * 1024 + tid;
        next[j] = e < nkeys ? counts[e] : 0;
      }
    }
    __syncthreads();
    int v[kItems];
    int local = 0;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      const int e = tid * kItems + j;
      v[j] = buf[e + (e >> 5)];
      local += v[j];
    }
    int x = local;
    for (int off = 1; off < 32; off <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, off);
      if (lane >= off) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int w = warp_sums[lane];
      for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, off);
        if (lane >= off) w += y;
      }
      warp_sums[lane] = w;
    }
    __syncthreads();
    int run = carry + x - local + (wid > 0 ? warp_sums[wid - 1] : 0);
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      const int e = tid * kItems + j;
      buf[e + (e >> 5)] = run;
      run += v[j];
    }
    if (tid == 1023) carry_s = run;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      const int e = j * 1024 + tid;
      if (base + e < nkeys) starts[base + e] = buf[e + (e >> 5)];
    }
    carry = carry_s;
    __syncthreads();  // buf and warp_sums are rewritten by the next round
  }
  if (tid == 0) starts[nkeys] = carry;
}

__global__ void k_scatter(const int* __restrict__ key, int n, const int* __restrict__ starts,
                          int* __restrict__ cursor, int* __restrict__ tmp) {
  chain_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = key[i];
  tmp[starts[k] + atomicAdd(&cursor[k], 1)] = i;
}

__global__ void k_rank(const int* __restrict__ key, int n, const int* __restrict__ starts,
                       const int* __restrict__ tmp, int* __restrict__ perm) {
  chain_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = key[i];
  const int b = starts[k], e = starts[k + 1];
  int r = 0;
  for (int j = b; j < e; ++j) r += tmp[j] < i;
  perm[b + r] = i;
}

// Box-sorted atoms: fractional coordinates and charge in FP64, and beside them
// the Cartesian position of the wrapped atom, x = s . lat, with the charge in
// FP32 for the real-space candidate test.
struct LatRows {
  double a[3][3];
};
__global__ void k_permute_box_seg(const BatchCell* __restrict__ cells,
                                  const int* __restrict__ prefix, int ncells, int n,
                                  const double4* __restrict__ in, const int* __restrict__ perm,
                                  double4* __restrict__ out, float4* __restrict__ x32) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const BatchCell& bc = cells[seg_cell(prefix, ncells, k)];  // sorted ranges = atom ranges
  const double4 v = in[perm[k]];
  out[k] = v;
  float c[3];
#pragma unroll
  for (int d = 0; d < 3; ++d)
    c[d] = static_cast<float>(v.x * bc.lat[0][d] + v.y * bc.lat[1][d] + v.z * bc.lat[2][d]);
  x32[k] = make_float4(c[0], c[1], c[2], static_cast<float>(v.w));
}

__global__ void k_permute_box(const double4* __restrict__ in, const int* __restrict__ perm, int n,
                              LatRows lat, double4* __restrict__ out, float4* __restrict__ x32) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double4 v = in[perm[k]];
  out[k] = v;
  float c[3];
#pragma unroll
  for (int d = 0; d < 3; ++d)
    c[d] = static_cast<float>(v.x * lat.a[0][d] + v.y * lat.a[1][d] + v.z * lat.a[2][d]);
  x32[k] = make_float4(c[0], c[1], c[2], static_cast<float>(v.w));
}

// ---------------------------------------------------------------------------
// Charge sums: per-CTA partials, then one CTA sums them in order.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  return v;
}

template <int NV>
__device__ void block_sum(double* v, double (*sh)[32]) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int j = 0; j < NV; ++j) v[j] = warp_sum(v[j]);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int j = 0; j < NV; ++j) sh[j][wid] = v[j];
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      double x = lane < nw ? sh[j][lane] : 0.0;
      v[j] = warp_sum(x);
    }
  }
}

__global__ void __launch_bounds__(256) k_charge_partial(const double* __restrict__ q, int n,
                                                        double* __restrict__ partial) {
  __shared__ double sh[3][32];
  double v[3] = {0.0, 0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double x = q[i];
    v[0] += x;
    v[1] += fabs(x);
    v[2] += x * x;
  }
  block_sum<3>(v, sh);
  if (threadIdx.x == 0)
    for (int j = 0; j < 3; ++j) partial[3 * blockIdx.x + j] = v[j];
}

__global__ void __launch_bounds__(256) k_sum_partials(const double* __restrict__ partial, int np,
                                                      int nv, double* __restrict__ out) {
  __shared__ double sh[6][32];
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (int i = threadIdx.x; i < np; i += blockDim.x)
    for (int j = 0; j < nv; ++j) v[j] += partial[static_cast<size_t>(nv) * i + j];
  block_sum<6>(v, sh);
  if (threadIdx.x == 0)
    for (int j = 0; j < nv; ++j) out[j] = v[j];
}

// ---------------------------------------------------------------------------
// Real-space pair sums.  One warp per (box-sorted) atom i; lanes take the
// candidates of each contiguous run of neighbour boxes 32 at a time.  The
// distance test is a prefilter in FP32 on Cartesian positions of the wrapped
// atoms (x_i - x_j - S lat, with the run's periodic shift S applied once per
// run), with a margin above its rounding error.  Only about one candidate in
// eight lies inside the cutoff, so the candidates that pass are first
// compacted into a per-warp queue in shared memory as (j, S); the warp then
// redoes, 32 queued pairs at a time with every lane busy, the separation
// ((s_i - s_j) - S) . lat, the cutoff test and the coincidence test in FP64
// from the fractional coordinates, as fft/ewald_fft_3d_real.f90:153-160 does,
// and evaluates the pair term (FP64, or FP32 in the mixed form: an FP32
// separation computed from Cartesian positions of up to a cell's size would
// lose too many digits at bonded distances).  The queue order, and so the
// summation order, is fixed by the candidate order: results are bitwise
// reproducible.
// ---------------------------------------------------------------------------
constexpr int kRealThreads = 256;
constexpr int kQueue = 64;  // per-warp queue: up to 31 carried over + 32 new

// One candidate as the scan hands it over.
struct Candidate {
  int j, sx, sy, sz;  // sorted index and periodic shift of j's run
  float r2;           // FP32 |x_i - x_j - S lat|^2
  bool valid;
};

template <class Pair, class Entry>
struct QueueBase {
  Entry* q;  // this warp's kQueue entries
  Pair& pair;
  int count = 0;
  __device__ __forceinline__ QueueBase(Entry* qbuf, Pair& p) : q(qbuf), pair(p) {}
  // Appends the lanes with take set, in lane order; runs a full batch of 32.
  template <class Eval>
  __device__ __forceinline__ void push(bool take, const Entry& e, Eval eval) {
    const int lane = threadIdx.x & 31;
    const unsigned m = __ballot_sync(0xffffffffu, take);
    if (take) q[count + __popc(m & ((1u << lane) - 1u))] = e;
    count += __popc(m);
    if (count >= 32) {
      __syncwarp();
      eval(q[lane]);
      __syncwarp();
      if (lane < count - 32) q[lane] = q[lane + 32];
      count -= 32;
      __syncwarp();
    }
  }
  template <class Eval>
  __device__ __forceinline__ void drain(Eval eval) {
    const int lane = threadIdx.x & 31;
    __syncwarp();
    if (lane < count) eval(q[lane]);
    count = 0;
  }
};

// Entries (j, S); at evaluation the separation, the exact cutoff test and the
// coincidence test are done in FP64.  F32TERM: the pair term then runs in FP32
// on the FP64 separation rounded once (the mixed form); otherwise in FP64.
template <class Pair, bool F32TERM>
struct PairQueue : QueueBase<Pair, int4> {
  const double4* __restrict__ srt;
  double4 ai;
  const RealGeom* g;
  double cut2;
  float pre2;  // FP32 prefilter bound: (r_cut + margin)^2
  __device__ __forceinline__ PairQueue(int4* qbuf, Pair& p, const double4* s, const double4& a,
                                       const RealGeom& geo, double c2, float p2)
      : QueueBase<Pair, int4>(qbuf, p), srt(s), ai(a), g(&geo), cut2(c2), pre2(p2) {}
  __device__ __forceinline__ void eval_entry(const int4& e) {
    const double4 aj = srt[e.x];
    const double d1 = (ai.x - aj.x) - e.y, d2 = (ai.y - aj.y) - e.z, d3 = (ai.z - aj.z) - e.w;
    double sep[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) sep[c] = d1 * g->lat[0][c] + d2 * g->lat[1][c] + d3 * g->lat[2][c];
    const double r2 = sep[0] * sep[0] + sep[1] * sep[1] + sep[2] * sep[2];
    if (r2 < 1.0e-24) this->pair.bad = 1;  // coincident charges
    if (r2 >= 1.0e-24 && r2 <= cut2) {
      if constexpr (F32TERM)
        this->pair.eval32(make_float4(static_cast<float>(sep[0]), static_cast<float>(sep[1]),
                                      static_cast<float>(sep[2]), static_cast<float>(aj.w)));
      else
        this->pair.eval(make_double4(sep[0], sep[1], sep[2], aj.w));
    }
  }
  __device__ __forceinline__ void operator()(const Candidate& c) {
    this->push(c.valid && c.r2 <= pre2, make_int4(c.j, c.sx, c.sy, c.sz),
               [this](const int4& e) { eval_entry(e); });
  }
  __device__ __forceinline__ void flush() {
    this->drain([this](const int4& e) { eval_entry(e); });
  }
};

template <class Visit>
__device__ __forceinline__ void for_each_candidate(const float4* __restrict__ x32,
                                                   const int* __restrict__ box_start, int k,
                                                   const double4& ai, const RealGeom& g,
                                                   Visit& visit) {
  const int lane = threadIdx.x & 31;
  int b[3];
  const double sv[3] = {ai.x, ai.y, ai.z};
  double xi[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    b[d] = min(static_cast<int>(sv[d] * g.nb[d]), g.nb[d] - 1);
    xi[d] = sv[0] * g.lat[0][d] + sv[1] * g.lat[1][d] + sv[2] * g.lat[2][d];
  }
  for (int dz = -g.R[2]; dz <= g.R[2]; ++dz) {
    const int bzr = b[2] + dz;
    const int sz = floor_div(bzr, g.nb[2]);
    const int wz = bzr - sz * g.nb[2];
    for (int dy = -g.R[1]; dy <= g.R[1]; ++dy) {
      const int byr = b[1] + dy;
      const int sy = floor_div(byr, g.nb[1]);
      const int wy = byr - sy * g.nb[1];
      int dx = -g.R[0];
      while (dx <= g.R[0]) {
        const int bxr = b[0] + dx;
        const int sx = floor_div(bxr, g.nb[0]);
        const int wx = bxr - sx * g.nb[0];
        const int len = min(g.R[0] - dx + 1, g.nb[0] - wx);
        const int first = (wz * g.nb[1] + wy) * g.nb[0] + wx;
        const int j0 = box_start[first], j1 = box_start[first + len];
        const bool home_image = (sx == 0 && sy == 0 && sz == 0);
        // x_i - S lat for this run, rounded once to FP32
        float base[3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
          base[d] = static_cast<float>(xi[d] - (sx * g.lat[0][d] + sy * g.lat[1][d] + sz * g.lat[2][d]));
        Candidate c;
        c.sx = sx;
        c.sy = sy;
        c.sz = sz;
        for (int jb = j0; jb < j1; jb += 32) {
          c.j = jb + lane;
          c.valid = c.j < j1 && !(home_image && c.j == k);
          c.r2 = 3.0e38f;
          if (c.valid) {
            const float4 xj = x32[c.j];
            const float d0 = base[0] - xj.x, d1 = base[1] - xj.y, d2 = base[2] - xj.z;
            c.r2 = fmaf(d0, d0, fmaf(d1, d1, d2 * d2));
          }
          visit(c);
        }
        dx += len;
      }
    }
  }
}

// Flat scan (RealGeom::flat).  The neighbourhood's rows (dy, dz) are laid out
// one per lane; each row is one or two contiguous runs of boxes (two when it
// wraps around the cell in x).  The non-empty runs go to a per-warp table in
// row order -- offset in the concatenated candidate list, sorted index of the
// first atom less that offset, the shift S and the run's x_i - S lat in FP32 --
// and the warp
// then walks the concatenated list 32 candidates at a time, so that a warp
// iteration is filled across run ends.  Rows, and the ends of rows, that lie
// wholly beyond the cutoff from atom i (by the distance from i to the boxes'
// slabs) are left out; the candidates visited keep the row-by-row scan's
// order, and the pairs inside the cutoff are the same.
constexpr int kRuns = 64;
struct RunTable {
  int start[kRuns + 1];  // offset of each run in the concatenated list; start[nrun] = total
  int4 info[kRuns];      // (j0 - start, sx, sy, sz): candidate v of run r is atom v + info.x
  float4 base[kRuns];    // x_i - S lat (w unused)
};

// Fractional distance from s to the slab [b / nb, (b + 1) / nb) of the
// unwrapped box index b (0 inside); inb = 1 / nb.
__device__ __forceinline__ double slab_gap(double s, int b, double inb) {
  const double lo = b * inb, hi = (b + 1) * inb;
  return s < lo ? lo - s : (s > hi ? s - hi : 0.0);
}

// reach2: squared cutoff with a relative margin far above the rounding of the
// slab distances; rows and boxes wholly beyond it are not visited.
template <class Visit>
__device__ __forceinline__ void for_each_candidate_flat(const float4* __restrict__ x32,
                                                        const int* __restrict__ box_start, int k,
                                                        const double4& ai, const RealGeom& g,
                                                        double reach2, RunTable& t,
                                                        Visit& visit) {
  const int lane = threadIdx.x & 31;
  int b[3];
  const double sv[3] = {ai.x, ai.y, ai.z};
  double xi[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    b[d] = min(static_cast<int>(sv[d] * g.nb[d]), g.nb[d] - 1);
    xi[d] = sv[0] * g.lat[0][d] + sv[1] * g.lat[1][d] + sv[2] * g.lat[2][d];
  }
  const int wdy = 2 * g.R[1] + 1;
  const int rows = wdy * (2 * g.R[2] + 1);
  // This lane's row: up to two runs.
  int j0[2] = {0, 0}, cnt[2] = {0, 0}, sx[2] = {0, 0}, sy = 0, sz = 0;
  if (lane < rows) {
    const int rz = (lane * g.rowmul) >> 16, ry = lane - rz * wdy;
    const int byr = b[1] + ry - g.R[1], bzr = b[2] + rz - g.R[2];
    sy = floor_div(byr, g.nb[1]);
    sz = floor_div(bzr, g.nb[2]);
    const int wy = byr - sy * g.nb[1], wz = bzr - sz * g.nb[2];
    // Distances from atom i to the row's y and z box slabs (normal to the
    // planes of constant s_y, s_z); the row region is the slabs' intersection.
    // With orthogonal plane normals its distance is sqrt(dy^2 + dz^2) and a
    // box of the row is reached when its x slab lies within
    // sqrt(reach^2 - dy^2 - dz^2); otherwise max(dy, dz) and reach bound them.
    const double dyz_y = slab_gap(sv[1], byr, g.inb[1]) * g.h[1];
    const double dyz_z = slab_gap(sv[2], bzr, g.inb[2]) * g.h[2];
    const double dperp2 = g.ortho ? dyz_y * dyz_y + dyz_z * dyz_z
                                  : fmax(dyz_y, dyz_z) * fmax(dyz_y, dyz_z);
    int dx = -g.R[0], dx_hi = g.R[0];
    if (dperp2 > reach2) {
      dx_hi = dx - 1;  // the whole row lies beyond the cutoff
    } else {
      const double fx = sqrt(g.ortho ? reach2 - dperp2 : reach2) * g.rl[0];
      dx = max(dx, static_cast<int>(floor((sv[0] - fx) * g.nb[0])) - b[0]);
      dx_hi = min(dx_hi, static_cast<int>(floor((sv[0] + fx) * g.nb[0])) - b[0]);
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (dx <= dx_hi) {
        const int bxr = b[0] + dx;
        const int s = floor_div(bxr, g.nb[0]);
        const int wx = bxr - s * g.nb[0];
        const int len = min(dx_hi - dx + 1, g.nb[0] - wx);
        const int first = (wz * g.nb[1] + wy) * g.nb[0] + wx;
        j0[h] = box_start[first];
        cnt[h] = box_start[first + len] - j0[h];
        sx[h] = s;
        dx += len;
      }
    }
  }
  // Compact the non-empty runs into the table in (row, run) order.
  const unsigned below = (1u << lane) - 1u;
  const unsigned m0 = __ballot_sync(0xffffffffu, cnt[0] > 0);
  const unsigned m1 = __ballot_sync(0xffffffffu, cnt[1] > 0);
  const int nrun = __popc(m0) + __popc(m1);
  int pos = __popc(m0 & below) + __popc(m1 & below);
  __syncwarp();
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    if (cnt[h] > 0) {
      t.info[pos] = make_int4(j0[h], sx[h], sy, sz);  // .x becomes j0 - start below
      t.start[pos] = cnt[h];  // counts for now; turned into offsets below
      float b3[3];
#pragma unroll
      for (int d = 0; d < 3; ++d)
        b3[d] = static_cast<float>(
            xi[d] - (sx[h] * g.lat[0][d] + sy * g.lat[1][d] + sz * g.lat[2][d]));
      t.base[pos] = make_float4(b3[0], b3[1], b3[2], 0.0f);
      ++pos;
    }
  }
  __syncwarp();
  // Exclusive prefix of the counts (entries lane and lane + 32).
  const int c0 = lane < nrun ? t.start[lane] : 0, c1 = lane + 32 < nrun ? t.start[lane + 32] : 0;
  int s0 = c0, s1 = c1;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int u0 = __shfl_up_sync(0xffffffffu, s0, off), u1 = __shfl_up_sync(0xffffffffu, s1, off);
    if (lane >= off) {
      s0 += u0;
      s1 += u1;
    }
  }
  const int half = __shfl_sync(0xffffffffu, s0, 31);
  const int total = half + __shfl_sync(0xffffffffu, s1, 31);
  __syncwarp();
  if (lane < nrun) {
    t.start[lane] = s0 - c0;
    t.info[lane].x -= s0 - c0;
  }
  if (lane + 32 < nrun) {
    t.start[lane + 32] = half + s1 - c1;
    t.info[lane + 32].x -= half + s1 - c1;
  }
  if (lane == 0) t.start[nrun] = total;
  __syncwarp();
  int rc = 0;  // the run holding the iteration's first candidate
  for (int v0 = 0; v0 < total; v0 += 32) {
    const int v = v0 + lane;
    Candidate c;
    c.j = 0;
    c.sx = c.sy = c.sz = 0;
    c.valid = false;
    c.r2 = 3.0e38f;
    if (v < total) {
      int r = rc;
      while (t.start[r + 1] <= v) ++r;
      const int4 e = t.info[r];
      c.j = v + e.x;
      c.sx = e.y;
      c.sy = e.z;
      c.sz = e.w;
      c.valid = !((e.y | e.z | e.w) == 0 && c.j == k);
      if (c.valid) {
        const float4 xj = x32[c.j];
        const float4 bs = t.base[r];
        const float d0 = bs.x - xj.x, d1 = bs.y - xj.y, d2 = bs.z - xj.z;
        c.r2 = fmaf(d0, d0, fmaf(d1, d1, d2 * d2));
      }
    }
    visit(c);
    while (rc + 1 < nrun && t.start[rc + 1] <= v0 + 32) ++rc;
  }
}

// FP32 prefilter bound for the FP64 cutoff test: the candidate separations
// carry a rounding error of a few FP32 ulps of the largest coordinate and
// shift, far below the margin.
inline float prefilter_bound(const RealGeom& g, double r_cut) {
  double extent = 0.0;
  for (int i = 0; i < 3; ++i) {
    double len = 0.0;
    for (int d = 0; d < 3; ++d) len += g.lat[i][d] * g.lat[i][d];
    extent += (2.0 * g.R[i] + 2.0) * std::sqrt(len);
  }
  const double r = r_cut + 1.0e-3 + 1.0e-5 * (extent + r_cut);
  return static_cast<float>(r * r);
}

// Pair term of fft/ewald_fft_3d_real.f90:153-172: FP64 (eval, FP64 separation),
// or its FP32 form (eval32, FP32 separation), accumulated in FP64.
struct EwaldPair {
  double alpha, qi;
  double pot = 0.0, f[3] = {0.0, 0.0, 0.0};
  int bad = 0;
  __device__ __forceinline__ void eval(const double4& e) {
    const double r2 = e.x * e.x + e.y * e.y + e.z * e.z;
    const double qj = e.w;
    const double r = sqrt(r2);
    const double rinv = 1.0 / r;
    const double ecr = erfc(alpha * r) * rinv;  // erfc(alpha r) / r
    pot += qj * ecr;
    const double ff =
        qi * qj * (2.0 * alpha / kSqrtPi * exp(-alpha * alpha * r2) + ecr) * (rinv * rinv);
    f[0] += ff * e.x;
    f[1] += ff * e.y;
    f[2] += ff * e.z;
  }
  __device__ __forceinline__ void eval32(const float4& e) {
    const float r2f = fmaf(e.x, e.x, fmaf(e.y, e.y, e.z * e.z));
    const float af = static_cast<float>(alpha);
    const float rinv = rsqrtf(r2f);
    const float r = r2f * rinv;
    const float ec = erfcf(af * r);
    const float pe = e.w * ec * rinv;
    pot += static_cast<double>(pe);
    const float ff = static_cast<float>(qi) * e.w *
                     (2.0f * af * 0.56418958354775628695f * expf(-af * af * r2f) + ec * rinv) *
                     (rinv * rinv);
    f[0] += static_cast<double>(ff * e.x);
    f[1] += static_cast<double>(ff * e.y);
    f[2] += static_cast<double>(ff * e.z);
  }
};

// Four CTAs of 256 threads per SM (64 registers): the candidate loads and the
// pair terms' dependent FP64 chains want the warps.
// The warp of sorted atom k (box_start: the cell's own box numbering).
template <bool MIXED>
__device__ __forceinline__ void real_space_body(const double4* __restrict__ srt,
                                                const float4* __restrict__ x32,
                                                const int* __restrict__ perm,
                                                const int* __restrict__ box_start, int k,
                                                const RealGeom& g, double alpha, double cut2,
                                                float pre2, double* __restrict__ pot,
                                                double* __restrict__ force,
                                                int* __restrict__ err) {
  __shared__ __align__(16) int4 queue[kRealThreads / 32][kQueue];
  __shared__ RunTable runs[kRealThreads / 32];
  const int lane = threadIdx.x & 31;
  const double4 ai = srt[k];
  EwaldPair pair;
  pair.alpha = alpha;
  pair.qi = ai.w;
  PairQueue<EwaldPair, MIXED> pq(queue[threadIdx.x >> 5], pair, srt, ai, g, cut2, pre2);
  if (g.flat)
    for_each_candidate_flat(x32, box_start, k, ai, g, cut2 * (1.0 + 1e-9), runs[threadIdx.x >> 5],
                              pq);
  else
    for_each_candidate(x32, box_start, k, ai, g, pq);
  pq.flush();
  // Transposed reduction of (pot, f_x, f_y, f_z): halves and quarters of the
  // warp each keep some of the four sums and pass the others on (6 shuffles of
  // doubles instead of 20); lanes 0, 8, 16, 24 end with the four totals.
  const bool hi16 = lane & 16, hi8 = lane & 8;
  const double s0 = hi16 ? pair.pot : pair.f[1], s1 = hi16 ? pair.f[0] : pair.f[2];
  const double k0 = hi16 ? pair.f[1] : pair.pot, k1 = hi16 ? pair.f[2] : pair.f[0];
  const double a0 = k0 + __shfl_xor_sync(0xffffffffu, s0, 16);
  const double a1 = k1 + __shfl_xor_sync(0xffffffffu, s1, 16);
  double t = (hi8 ? a1 : a0) + __shfl_xor_sync(0xffffffffu, hi8 ? a0 : a1, 8);
  t += __shfl_xor_sync(0xffffffffu, t, 4);
  t += __shfl_xor_sync(0xffffffffu, t, 2);
  t += __shfl_xor_sync(0xffffffffu, t, 1);
  const int bad = __any_sync(0xffffffffu, pair.bad);
  if ((lane & 7) == 0) {
    const int i = perm[k];
    const int c = lane >> 3;  // 0: pot, 1..3: force component c - 1
    if (c == 0)
      pot[i] = t;
    else
      force[3 * i + c - 1] = t;
    if (c == 0 && bad) atomicOr(err, 1);
  }
}

template <bool MIXED>
__global__ void __launch_bounds__(kRealThreads, 4) k_real_space(const double4* __restrict__ srt,
                                                             const float4* __restrict__ x32,
                                                             const int* __restrict__ perm,
                                                             const int* __restrict__ box_start,
                                                             int n, RealGeom g, double alpha,
                                                             double cut2, float pre2,
                                                             double* __restrict__ pot,
                                                             double* __restrict__ force,
                                                             int* __restrict__ err) {
  const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (k >= n) return;
  real_space_body<MIXED>(srt, x32, perm, box_start, k, g, alpha, cut2, pre2, pot, force, err);
}

// Every cell of a batch: the warp's atom k picks its cell's cell-list geometry,
// splitting and cutoff; a coincident pair flags the cell (err[cell]).
template <bool MIXED>
__global__ void __launch_bounds__(kRealThreads, 4) k_real_space_seg(
    const BatchCell* __restrict__ cells, const int* __restrict__ prefix, int ncells,
    const double4* __restrict__ srt, const float4* __restrict__ x32, const int* __restrict__ perm,
    const int* __restrict__ box_start, int n, double* __restrict__ pot,
    double* __restrict__ force, int* __restrict__ err) {
  const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (k >= n) return;
  const int c = seg_cell(prefix, ncells, k);
  const BatchCell& bc = cells[c];
  const RealGeom g = bc.rg;
  real_space_body<MIXED>(srt, x32, perm, box_start + bc.box0, k, g, bc.alpha, bc.cut2, bc.pre2,
                         pot, force, err + c);
}

// Real-space virial of invRStress with addNeighbourContribsStress
// (coulomb.F90:2836-2905).  Over the full list with a factor 1/2 (the half
// list's pairs each appear twice), r (x) f + f (x) r with f = derivRTerm(r) q_i q_j
// collapses to derivRTerm-scalar * q_i q_j * r (x) r.
struct StressPair {
  double alpha, qi;
  double s[6] = {0, 0, 0, 0, 0, 0};  // xx, yy, zz, xy, xz, yz
  int bad = 0;
  __device__ __forceinline__ void eval(const double4& e) {
    const double d2 = e.x * e.x + e.y * e.y + e.z * e.z;
    const double rr = sqrt(d2);
    const double fac = alpha * rr;
    const double dr = (-2.0 / kSqrtPi * exp(-fac * fac) * fac - erfc(fac)) / (rr * rr * rr);
    const double w = dr * qi * e.w;
    s[0] += w * e.x * e.x;
    s[1] += w * e.y * e.y;
    s[2] += w * e.z * e.z;
    s[3] += w * e.x * e.y;
    s[4] += w * e.x * e.z;
    s[5] += w * e.y * e.z;
  }
};

__global__ void __launch_bounds__(kRealThreads) k_real_stress(const double4* __restrict__ srt,
                                                              const float4* __restrict__ x32,
                                                              const int* __restrict__ box_start,
                                                              int n, RealGeom g, double alpha,
                                                              double cut2, float pre2,
                                                              double* __restrict__ partial6,
                                                              int* __restrict__ err) {
  __shared__ __align__(16) int4 queue[kRealThreads / 32][kQueue];
  __shared__ RunTable runs[kRealThreads / 32];
  const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (k >= n) return;
  const double4 ai = srt[k];
  StressPair pair;
  pair.alpha = alpha;
  pair.qi = ai.w;
  PairQueue<StressPair, false> pq(queue[threadIdx.x >> 5], pair, srt, ai, g, cut2, pre2);
  if (g.flat)
    for_each_candidate_flat(x32, box_start, k, ai, g, cut2 * (1.0 + 1e-9), runs[threadIdx.x >> 5],
                              pq);
  else
    for_each_candidate(x32, box_start, k, ai, g, pq);
  pq.flush();
#pragma unroll
  for (int j = 0; j < 6; ++j) pair.s[j] = warp_sum(pair.s[j]);
  const int bad = __any_sync(0xffffffffu, pair.bad);
  if (lane == 0) {
#pragma unroll
    for (int j = 0; j < 6; ++j) partial6[6 * static_cast<size_t>(k) + j] = pair.s[j];
    if (bad) atomicOr(err, 1);
  }
}

// ---------------------------------------------------------------------------
// Structure factors: one CTA per wave vector.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_structure_factors(const double* __restrict__ x,
                                                           const double* __restrict__ q, int n,
                                                           const double* __restrict__ kvec,
                                                           double* __restrict__ out) {
  __shared__ double sh[2][32];
  const int v = blockIdx.x;
  const double kx = kvec[3 * v], ky = kvec[3 * v + 1], kz = kvec[3 * v + 2];
  double acc[2] = {0.0, 0.0};
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double ph = kx * x[3 * i] + ky * x[3 * i + 1] + kz * x[3 * i + 2];
    double sn, cs;
    sincos(ph, &sn, &cs);
    acc[0] += q[i] * cs;
    acc[1] += q[i] * sn;
  }
  block_sum<2>(acc, sh);
  if (threadIdx.x == 0) {
    out[2 * v] = acc[0];
    out[2 * v + 1] = acc[1];
  }
}

// Reciprocal part of invRStress (coulomb.F90:2800-2833) per half-space G: the
// reference visits +G and -G separately; |S(-G)| = |S(G)| and the tensor is
// even in G, so both visits are 2 x the +G term.
__global__ void k_recip_stress(const double* __restrict__ kvec, const double* __restrict__ sk,
                               int nk, double alpha, double* __restrict__ partial6) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nk) return;
  const double g[3] = {kvec[3 * v], kvec[3 * v + 1], kvec[3 * v + 2]};
  const double sr = sk[2 * v], si = sk[2 * v + 1];
  const double a2 = alpha * alpha;
  const double g2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
  const double im = 2.0 * (sr * sr + si * si) * exp(-g2 / (4.0 * a2)) / g2;
  const double c = 2.0 * (1.0 / (4.0 * a2) + 1.0 / g2);
  partial6[6 * v + 0] = (1.0 - c * g[0] * g[0]) * im;
  partial6[6 * v + 1] = (1.0 - c * g[1] * g[1]) * im;
  partial6[6 * v + 2] = (1.0 - c * g[2] * g[2]) * im;
  partial6[6 * v + 3] = -c * g[0] * g[1] * im;
  partial6[6 * v + 4] = -c * g[0] * g[2] * im;
  partial6[6 * v + 5] = -c * g[1] * g[2] * im;
}

// Direct Fourier sum of ewald_direct_3d: thread per atom, loop over modes.
__global__ void __launch_bounds__(256) k_direct_kspace(const double* __restrict__ x,
                                                       const double* __restrict__ q, int n,
                                                       const double* __restrict__ kvec,
                                                       const double* __restrict__ wk,
                                                       const double* __restrict__ sk, int nk,
                                                       double* __restrict__ pot,
                                                       double* __restrict__ force) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2];
  double p = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
  for (int v = 0; v < nk; ++v) {
    const double kx = kvec[3 * v], ky = kvec[3 * v + 1], kz = kvec[3 * v + 2];
    double sn, cs;
    sincos(kx * xi + ky * yi + kz * zi, &sn, &cs);
    const double sr = sk[2 * v], si = sk[2 * v + 1];
    const double lr = sr * cs + si * sn;
    const double li = si * cs - sr * sn;
    p += wk[v] * lr;
    const double ff = wk[v] * li;
    fx -= ff * kx;
    fy -= ff * ky;
    fz -= ff * kz;
  }
  pot[i] += p;
  if (force) {
    force[3 * i] += q[i] * fx;
    force[3 * i + 1] += q[i] * fy;
    force[3 * i + 2] += q[i] * fz;
  }
}

inline int blocks_for(long n, int threads) { return static_cast<int>((n + threads - 1) / threads); }

}  // namespace

void launch_atom_prep(const double* pos, long sa, long sd, const double* q, int n, const Cell& cell,
                      const int nb[3], const int ngrid[3], double4* s4, int* box_key,
                      int4* mesh_c, double4* mesh_fr, cudaStream_t st) {
  if (n == 0) return;
  PrepArgs a;
  for (int i = 0; i < 3; ++i) {
    for (int d = 0; d < 3; ++d) a.rec[i][d] = cell.rec[i][d];
    a.nb[i] = nb ? nb[i] : 0;
    a.ng[i] = ngrid ? ngrid[i] : 0;
  }
  k_atom_prep<<<blocks_for(n, 256), 256, 0, st>>>(pos, sa, sd, q, n, a, s4, box_key, mesh_c,
                                                  mesh_fr);
  ++g_launches;
}

void launch_bucket_sort(const int* key, int n, int nkeys, int* counts, int* cursor, int* starts,
                        int* tmp, int* perm, cudaStream_t st) {
  cudaMemsetAsync(counts, 0, sizeof(int) * nkeys, st);
  cudaMemsetAsync(cursor, 0, sizeof(int) * nkeys, st);
  if (n > 0) {
    k_count<<<blocks_for(n, 256), 256, 0, st>>>(key, n, counts);
    ++g_launches;
  }
  if (n > 0)
    launch_chained(k_scan, 1, 1024, 0, st, counts, nkeys, starts);
  else  // the stream's previous operation is a memset
    k_scan<<<1, 1024, 0, st>>>(counts, nkeys, starts);
  ++g_launches;
  if (n > 0) {
    launch_chained(k_scatter, blocks_for(n, 256), 256, 0, st, key, n, starts, cursor, tmp);
    launch_chained(k_rank, blocks_for(n, 256), 256, 0, st, key, n, starts, tmp, perm);
    g_launches += 2;
  }
}

void launch_scan(const int* counts, int nkeys, int* starts, bool after_kernel, cudaStream_t st) {
  if (after_kernel)
    launch_chained(k_scan, 1, 1024, 0, st, counts, nkeys, starts);
  else
    k_scan<<<1, 1024, 0, st>>>(counts, nkeys, starts);
  ++g_launches;
}

void launch_permute_box(const double4* in, const int* perm, int n, const double (*lat)[3],
                        double4* out, float4* x32, cudaStream_t st) {
  if (n == 0) return;
  LatRows L;
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) L.a[i][d] = lat[i][d];
  k_permute_box<<<blocks_for(n, 256), 256, 0, st>>>(in, perm, n, L, out, x32);
  ++g_launches;
}

void launch_charge_sums(const double* q, int n, double* partial, double* out, cudaStream_t st) {
  const int blocks = 148;
  k_charge_partial<<<blocks, 256, 0, st>>>(q, n, partial);
  k_sum_partials<<<1, 256, 0, st>>>(partial, blocks, 3, out);
  g_launches += 2;
}

void launch_real_space(const double4* srt, const float4* x32, const int* perm,
                       const int* box_start, int n, const RealGeom& g, double alpha, double r_cut,
                       int mixed, double* pot, double* force, int* err, cudaStream_t st) {
  if (n == 0) return;
  const int blocks = blocks_for(static_cast<long>(n) * 32, kRealThreads);
  const float pre2 = prefilter_bound(g, r_cut);
  if (mixed)
    k_real_space<true><<<blocks, kRealThreads, 0, st>>>(srt, x32, perm, box_start, n, g, alpha,
                                                        r_cut * r_cut, pre2, pot, force, err);
  else
    k_real_space<false><<<blocks, kRealThreads, 0, st>>>(srt, x32, perm, box_start, n, g, alpha,
                                                         r_cut * r_cut, pre2, pot, force, err);
  ++g_launches;
}

void launch_atom_prep_seg(const BatchLaunch& b, const double* coords3n, const double* q,
                          double4* s4, int* box_key, int4* mesh_c, double4* mesh_fr,
                          cudaStream_t st) {
  if (b.n_atoms == 0) return;
  k_atom_prep_seg<<<blocks_for(b.n_atoms, 256), 256, 0, st>>>(
      b.cells, b.p_atoms, b.ncells, b.n_atoms, coords3n, q, s4, box_key, mesh_c, mesh_fr);
  ++g_launches;
}

void launch_permute_box_seg(const BatchLaunch& b, const double4* in, const int* perm,
                            double4* out, float4* x32, cudaStream_t st) {
  if (b.n_atoms == 0) return;
  k_permute_box_seg<<<blocks_for(b.n_atoms, 256), 256, 0, st>>>(b.cells, b.p_atoms, b.ncells,
                                                                b.n_atoms, in, perm, out, x32);
  ++g_launches;
}

void launch_real_space_seg(const BatchLaunch& b, const double4* s4s, const float4* x32,
                           const int* perm, const int* box_start, double* pot, double* force,
                           int* cell_err, cudaStream_t st) {
  if (b.n_atoms == 0) return;
  const int blocks = blocks_for(static_cast<long>(b.n_atoms) * 32, kRealThreads);
  if (b.mixed)
    k_real_space_seg<true><<<blocks, kRealThreads, 0, st>>>(b.cells, b.p_atoms, b.ncells, s4s, x32,
                                                            perm, box_start, b.n_atoms, pot,
                                                            force, cell_err);
  else
    k_real_space_seg<false><<<blocks, kRealThreads, 0, st>>>(b.cells, b.p_atoms, b.ncells, s4s,
                                                             x32, perm, box_start, b.n_atoms, pot,
                                                             force, cell_err);
  ++g_launches;
}

float real_prefilter_bound(const RealGeom& g, double r_cut) { return prefilter_bound(g, r_cut); }

void launch_real_stress(const double4* srt, const float4* x32, const int* box_start, int n,
                        const RealGeom& g, double alpha, double max_r, double* partial6,
                        double* out6, int* err, cudaStream_t st) {
  if (n == 0) return;
  k_real_stress<<<blocks_for(static_cast<long>(n) * 32, kRealThreads), kRealThreads, 0, st>>>(
      srt, x32, box_start, n, g, alpha, max_r * max_r, prefilter_bound(g, max_r), partial6, err);
  k_sum_partials<<<1, 256, 0, st>>>(partial6, n, 6, out6);
  g_launches += 2;
}

void launch_sum_partials(const double* partial, int np, int nv, double* out, cudaStream_t st) {
  k_sum_partials<<<1, 256, 0, st>>>(partial, np, nv, out);
  ++g_launches;
}

void launch_structure_factors(const double* coords3n, const double* q, int n, const double* kvec,
                              int nk, double* out, cudaStream_t st) {
  if (nk == 0) return;
  k_structure_factors<<<nk, 256, 0, st>>>(coords3n, q, n, kvec, out);
  ++g_launches;
}

void launch_recip_stress(const double* kvec, const double* sk, int nk, double alpha,
                         double* partial6, double* out6, cudaStream_t st) {
  if (nk > 0) {
    k_recip_stress<<<blocks_for(nk, 256), 256, 0, st>>>(kvec, sk, nk, alpha, partial6);
    ++g_launches;
  }
  k_sum_partials<<<1, 256, 0, st>>>(partial6, nk, 6, out6);
  ++g_launches;
}

void launch_direct_kspace(const double* coords3n, const double* q, int n, const double* kvec,
                          const double* wk, const double* sk, int nk, double* pot, double* force,
                          cudaStream_t st) {
  if (n == 0 || nk == 0) return;
  k_direct_kspace<<<blocks_for(n, 256), 256, 0, st>>>(coords3n, q, n, kvec, wk, sk, nk, pot, force);
  ++g_launches;
}

}  // namespace ewg
