// ewg_kernels.h -- host-callable launchers of the Ewald kernels.
#pragma once

#include <cuda_runtime.h>

#include "ewg_internal.h"

namespace ewg {

// Launch counter shared by every launcher (the context copies it out).
extern thread_local long long g_launches;

// Programmatic dependent launch along the evaluation's chain of short kernels.
// A chained kernel starts with chain_enter(): griddepcontrol.wait holds every
// thread until the previous grid on the stream has completed and its writes
// are visible (a no-op for a kernel launched without the attribute), so the
// kernel touches no global memory before its predecessor is done; then
// launch_dependents lets the next grid's CTAs be placed on the SMs this grid's
// last wave leaves idle, instead of after a launch gap.
__device__ __forceinline__ void chain_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Launch a chained kernel; the stream's previous operation must be a kernel.
template <typename... P, typename... A>
void launch_chained(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                    A&&... args) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, static_cast<A&&>(args)...);
}

// Stages of one evaluation, for the per-stage device timing.
enum Stage {
  ST_PREP, ST_REAL, ST_WEIGHTS, ST_SPREAD, ST_FFT_X_R2C, ST_FFT_Y_FWD, ST_FFT_Z_INFL,
  ST_FFT_Y_INV, ST_FFT_X_C2R, ST_GATHER, ST_COUNT
};

// Event marks on one stream; the interval after mark i belongs to tag[i].
struct Profiler {
  static constexpr int kMax = 64;
  bool on = false;
  int n = 0;
  cudaEvent_t ev[kMax] = {};
  int tag[kMax] = {};
  double ms[ST_COUNT] = {};
  long long launches[ST_COUNT] = {};
  long long launch_mark[kMax] = {};
};
// Close the running interval and open one for `stage` (-1: none).
void prof_mark(Profiler* p, cudaStream_t st, int stage);
// After the stream is synchronised: fold the intervals into ms[] and reset.
void prof_collect(Profiler* p);

// ---- atoms: fractional coordinates, keys, sorting (ewg_real.cu) ----------

// Per atom: wrapped fractional coordinates s and charge (double4), real-space
// box key, mesh lowest point and fraction (nfft/nfft.f90:122-159).  Null
// outputs (and null nb / ngrid) are skipped.
// positions: element (i, d) at pos[i * sa + d * sd].
void launch_atom_prep(const double* pos, long sa, long sd, const double* q, int n, const Cell& cell,
                      const int nb[3], const int ngrid[3], double4* s4, int* box_key, int4* mesh_c,
                      double4* mesh_fr, cudaStream_t st);

// Stable counting sort by key: perm[k] = atom with the k-th key in (key, index)
// order; starts[nkeys + 1] are bucket offsets.  Scratch: counts/cursor (nkeys),
// tmp (n).
void launch_bucket_sort(const int* key, int n, int nkeys, int* counts, int* cursor, int* starts,
                        int* tmp, int* perm, cudaStream_t st);

// Exclusive scan of counts[0..nkeys) into starts[0..nkeys] (one CTA), chained
// to the stream's previous kernel when after_kernel.
void launch_scan(const int* counts, int nkeys, int* starts, bool after_kernel, cudaStream_t st);

// Box-sorted atoms: out[k] = in[perm[k]] (fractional s, q) and x32[k] the
// Cartesian position s . lat with q, in FP32, for the real-space distance test.
void launch_permute_box(const double4* in, const int* perm, int n, const double (*lat)[3],
                        double4* out, float4* x32, cudaStream_t st);

// Charge sums for the parameter chain on device-resident charges:
// out[0] = sum q, out[1] = sum |q|, out[2] = sum q^2 (fixed-order reduction).
void launch_charge_sums(const double* q, int n, double* partial, double* out, cudaStream_t st);

// Real-space erfc pair sum (fft/ewald_fft_3d_real.f90:81-187 and
// direct/ewald_direct_3d.f90:192-309) over box-sorted atoms.  Writes pot and
// force (3,N) by original atom index.  mixed != 0 evaluates the pair terms in
// FP32 and accumulates in FP64.
void launch_real_space(const double4* s4_sorted, const float4* x32_sorted, const int* perm,
                       const int* box_start, int n, const RealGeom& g, double alpha, double r_cut,
                       int mixed, double* pot, double* force, int* err, cudaStream_t st);

// Real-space virial of invRStress (coulomb.F90:2836-2905): per-atom partial
// tensors (6 per atom) then a fixed-order sum into out6.
// Fixed-order sum of np partial vectors of nv doubles (one CTA).
void launch_sum_partials(const double* partial, int np, int nv, double* out, cudaStream_t st);
void launch_real_stress(const double4* s4_sorted, const float4* x32_sorted, const int* box_start,
                        int n, const RealGeom& g, double alpha, double max_r, double* partial6,
                        double* out6, int* err, cudaStream_t st);

// Structure factors S(k) = sum_j q_j exp(i k . x_j) for a list of Cartesian
// wave vectors; x(3,N) atom-major Cartesian coordinates.  out: 2 per vector.
void launch_structure_factors(const double* coords3n, const double* q, int n, const double* kvec,
                              int nk, double* out, cudaStream_t st);

// Reciprocal stress of invRStress (coulomb.F90:2800-2833) from S(G):
// per-vector tensors then a fixed-order sum into out6.
void launch_recip_stress(const double* kvec, const double* sk, int nk, double alpha,
                         double* partial6, double* out6, cudaStream_t st);

// Direct Fourier sum of the direct engine (direct/ewald_direct_3d.f90:131-174):
// pot[i] += sum_k w_k Re(S(k) e^{-ik.x_i}), force[i] -= q_i w_k Im(...) k.
void launch_direct_kspace(const double* coords3n, const double* q, int n, const double* kvec,
                          const double* wk, const double* sk, int nk, double* pot, double* force,
                          cudaStream_t st);

// ---- mesh (ewg_mesh.cu) ----------------------------------------------------

// Tile shape of the spread and gather (points along x, y, z).
constexpr int kTileX = 8, kTileY = 8, kTileZ = 8;

// Geometry of the particle-side stencil work.
struct StencilDims {
  int n[3];        // fine grid
  int T[3];        // tile edge per axis
  int ntiles[3];   // tiles per axis
  int S[3];        // most tiles one stencil touches per axis
  int woff[3];     // per-atom weight offsets per axis
  int wstride;     // per-atom weight count: sum S_d T_d
  int m;           // window half-width
  double b;        // window shape
  double pref;     // 1/sqrt(pi b)
  int ad;          // 1: window derivatives stored after the weights (forces by
                   // analytic differentiation of the window)
  int dwoff;       // per-atom offset of the derivative rows (woff[d] + dwoff)
  int pstride;     // gather partials per atom: S_x S_y S_z slots (or more, when
                   // cells of a batch share one layout)
};

// Everything the mesh pipeline needs, resolved on the host.
struct MeshPlan {
  MeshGeom g;
  StencilDims sd;
  FftPlan fft[3];
  int mixed;                      // 0: FP64, 1: FP32 storage/products
  int lines_cap = 0;              // most FFT lines per CTA (0: the most that fit)
  int gather_warps = 4;           // FP64 i k gather CTA: 2, 4 or 8 warps
  int stencil = 1;                // mixed form's spread and gather: 1 FP64 tensor
                                  // cores on FP32 data, 2 FP32 CUDA cores
  Profiler* prof = nullptr;
  const double* corr2[3] = {nullptr, nullptr, nullptr};  // squared deconvolution factors, index k + H
};

// ---- segmented launches of the batched form --------------------------------
// The cells of a batch lie end to end: their atoms in global arrays (the
// caller's CSR order, and after the global box sort, cell by cell in box
// order), their cell-list boxes and mesh tiles as consecutive key ranges of
// global counting sorts, their grids in separate buffers.  One launch per
// stage covers every cell; its global index (atom, work item or block) maps to
// its cell through the launch's prefix array (prefix[c] = first index of cell
// c, prefix[ncells] = total), and the cell's parameters come from the device
// table below.
struct BatchCell {
  int atom0, natoms;  // global atom range
  int box0, tile0;    // first key of the cell in the global box and tile sorts
  double lat[3][3], rec[3][3];
  RealGeom rg;
  double alpha, cut2;
  float pre2;
  double self_coef;
  MeshGeom g;
  StencilDims sd;
  FftPlan fft[3];
  const double* corr2[3];
  void *grid, *A1, *A2, *B2, *B1, *out;
};

// The cell holding global index idx: the last c with prefix[c] <= idx (cells
// with no work in a launch have prefix[c] == prefix[c + 1] and are skipped).
__device__ __forceinline__ int seg_cell(const int* __restrict__ prefix, int ncells, long idx) {
  int lo = 0, hi = ncells - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= idx)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Host description of one segmented batch: the device table, the prefix
// array of every launch (device) and the totals (host).
struct BatchLaunch {
  const BatchCell* cells = nullptr;
  int ncells = 0;
  int mixed = 0, nc = 1, nparts = 1, ad = 0;
  int L = 1;           // FFT lines per CTA, one value for every cell
  int uniform[3] = {0, 0, 0};  // every cell has the same length along this axis
  FftPlan plan[3];             // that length's plan (when uniform)
  size_t smem[3] = {0, 0, 0};  // FFT pass shared memory per axis (the largest cell's)
  size_t smem_z = 0;
  int lpa = 32;        // lanes per atom of the final sum
  // prefix arrays (device) and totals
  const int* p_atoms = nullptr;   int n_atoms = 0;
  const int* p_weights = nullptr; long n_weights = 0;  // natoms (S_x + S_y + S_z)
  const int* p_slots = nullptr;   long n_slots = 0;    // natoms S_x S_y S_z
  const int* p_tiles = nullptr;   int n_tiles = 0;
  const int* p_r2c = nullptr;     int n_r2c = 0;
  const int* p_yfwd = nullptr;    int n_yfwd = 0;
  const int* p_z = nullptr;       int n_z = 0;
  const int* p_yinv = nullptr;    int n_yinv = 0;
  const int* p_c2r = nullptr;     int n_c2r = 0;
  const int* p_final = nullptr;   long n_final = 0;    // natoms lpa
  int n_boxes = 0;
};

// Segmented counterparts of the single-cell launchers (same work per cell).
void launch_atom_prep_seg(const BatchLaunch& b, const double* coords3n, const double* q,
                          double4* s4, int* box_key, int4* mesh_c, double4* mesh_fr,
                          cudaStream_t st);
void launch_permute_box_seg(const BatchLaunch& b, const double4* in, const int* perm,
                            double4* out, float4* x32, cudaStream_t st);
void launch_real_space_seg(const BatchLaunch& b, const double4* s4s, const float4* x32,
                           const int* perm, const int* box_start, double* pot, double* force,
                           int* cell_err, cudaStream_t st);
void launch_weights_seg(const BatchLaunch& b, const int4* mesh_c, const double4* mesh_fr,
                        const int* perm, void* wtab, void* qk, int4* slot, cudaStream_t st);
void launch_pair_bins_seg(const BatchLaunch& b, const int4* slot, int* counts, int* cursor,
                          int* tile_start, int4* tmp, int2* pairs, cudaStream_t st);
void launch_spread_seg(const BatchLaunch& b, const int* tile_start, const int2* pairs,
                       const void* wtab, const void* qk, cudaStream_t st);
void launch_forward_and_weight_seg(const BatchLaunch& b, cudaStream_t st);
void launch_inverse_seg(const BatchLaunch& b, cudaStream_t st);
void launch_gather_seg(const BatchLaunch& b, const int* tile_start, const int2* pairs,
                       const void* wtab, double* part, cudaStream_t st);
void launch_gather_final_seg(const BatchLaunch& b, const int4* slot, const int* perm,
                             const double* part, const double* q, const double* pot_sr,
                             const double* f_sr, double* pot, double* force, cudaStream_t st);
// FP32 prefilter bound of the real-space distance test for this geometry.
float real_prefilter_bound(const RealGeom& g, double r_cut);
// FFT lines per CTA a pass of length n (plus `extra` elements per line) would
// take alone, and the shared bytes of such a pass at L lines.
int mesh_batch_lines(int n, bool mixed, int extra);
// Blocks per cell of each pass (x R2C, y forward, z, y inverse, x C2R) at L
// lines per CTA and nc grids through the inverse passes.
void mesh_pass_blocks(const MeshGeom& g, int L, int nc, int out[5]);
size_t mesh_pass_smem(int n, int L, bool mixed, int extra);

// Tiled window weights per sorted atom (wtab: wstride values per atom), slot
// origin and count per axis (slot: first | count << 16 in x, y, z), and the
// charges in sorted order (qk).  mesh_c / mesh_fr are in atom order and are
// read through the permutation (sorted atom k is atom perm[k]; the cell-list
// box order, which keeps neighbouring atoms close in the tables).
void launch_weights(const MeshPlan& mp, const int4* mesh_c, const double4* mesh_fr,
                    const int* perm, int n, void* wtab, void* qk, int4* slot, cudaStream_t st);

// Only the charges in sorted order, qk[k] = q[perm[k]] (FP32 in the mixed form):
// the resident path's refresh when the geometry and so the weights and the
// pair lists are unchanged.
void launch_sorted_charges(const MeshPlan& mp, const double* q, const int* perm, int n, void* qk,
                           cudaStream_t st);

// Bins every (atom, tile) pair by tile, buckets ordered by atom index:
// pairs[tile_start[t] .. tile_start[t+1]) = (atom, packed slot).  Scratch:
// counts/cursor (ntiles), tmp (npairs_max); npairs_max = n * S_x * S_y * S_z.
void launch_pair_bins(const MeshPlan& mp, const int4* slot, int n, int* counts, int* cursor,
                      int* tile_start, int4* tmp, int2* pairs, int npairs_max, cudaStream_t st);

// Tile-owned deterministic spread (adjoint_nfft_3d step 1, nfft/nfft.f90:253-278).
void launch_spread(const MeshPlan& mp, const int* tile_start, const int2* pairs, const void* wtab,
                   const void* qk, void* grid, cudaStream_t st);

// Pruned forward transform of the real grid to the compact spectrum, fused with
// the influence weights and the first inverse pass: grid -> A1 -> A2 -> B2.
// nc = 1 (potential) or 4 (potential and its three fractional derivatives
// d/ds_d; B2 then holds two spectra, B1 three, the output four real grids).
// stress_part (optional, K1 x K2 x 6 doubles, zeroed): per-CTA partials of the
// reciprocal strain derivative, accumulated by the z pass.
void launch_forward_and_weight(const MeshPlan& mp, const void* grid, void* A1, void* A2, void* B2,
                               int nc, cudaStream_t st, double* stress_part = nullptr);

// Remaining inverse passes B2 -> B1 -> interleaved real grids (nc per point).
void launch_inverse(const MeshPlan& mp, const void* B2, void* B1, void* out, int nc, cudaStream_t st);

// Gather (forward_nfft_3d step 3, nfft/nfft.f90:380-402): per-(atom, tile)
// partial sums of the nc interleaved real grids into part (nslots * nc per atom).
// With mp.sd.ad and force wanted, the grid holds the potential alone (nc = 1)
// and the partials are four: the potential and its derivatives along the three
// fractional coordinates (window derivatives times the grid).
void launch_gather(const MeshPlan& mp, const int* tile_start, const int2* pairs, const void* wtab,
                   const void* out_grid, int nc, double* part, cudaStream_t st);

// Fixed-order sum of each atom's partials with the final assembly
// (fft/ewald_fft_3d.f90:121-132): pot = (sr + lr) + self, force = sr + q lr.
// nparts = 1 or 4.  rec (nullptr for ik partials): the dual basis rows b_d;
// the partials are then fractional derivatives D_d and the long-range force
// is -q sum_d D_d b_d.
void launch_gather_final(const MeshPlan& mp, const int4* slot, const int* mesh_perm,
                         const double* part, int nparts, int n, const double* q_orig,
                         double self_coef, double pot_shift, const double* pot_sr,
                         const double* force_sr, double* pot, double* force,
                         const double (*rec)[3], cudaStream_t st);

// Device byte sizes of the mesh buffers (nc grid components, nparts partials
// per (atom, slot)).
struct MeshSizes {
  size_t grid, A1, A2, B2, B1, out, wtab, qk, slot, part;
};
MeshSizes mesh_sizes(const MeshGeom& g, const StencilDims& sd, int mixed, int nc, int natoms,
                     int nparts);

// Shared-memory limits of the FFT and gather kernels (once per device).
// Stock Ewald lattice sums for potentials and gradients at arbitrary points
// (ewg_external.cu): cell translations R (origin first), half-space reciprocal
// vectors G (Cartesian, with 2 pi) and the other group's structure factors
// sf[2g] = sum q cos(G.r), sf[2g+1] = sum q sin(G.r); all device pointers.
struct ExtLattice {
  const double* R;
  int nR;
  const double* G;
  int nG;
  const double* sf;
  double alpha, volume;
};
void launch_ext_potential(int nt, const double* tc, int ns, const double* sc, const double* sq,
                          const double* blur, double eps2, const ExtLattice& L, double const_term,
                          double* pot, cudaStream_t st);
void launch_ext_gradient(int nt, const double* tc, int ns, const double* sc, const double* sq,
                         const double* blur, const ExtLattice& L, const double* scale,
                         double* grad, cudaStream_t st);
void launch_ext_source_gradient(int nt, const double* tc, const double* tq, int ns,
                                const double* sc, const double* sq, const double* blur,
                                const ExtLattice& L, double* grad, cudaStream_t st);

// Real-space half of the mesh-based point potentials (ewg_points.cu): per
// target, the pair terms of ewaldReal / derivEwaldReal (dftb/coulomb.F90:2520-2625)
// with splitting alpha over the sources within r_cut (cell list of the
// sources in box order, periodic images included), plus the self term of
// coincident points.  Writes pot (nt) and/or grad (3, nt) when asked.
struct PointsReal {
  int nb[3];        // source boxes per axis
  int R[3];         // neighbour box range per axis
  double lat[3][3];
  double rec[3][3];
  double r_cut2;
  double alpha;
  int want_pot, want_grad;
};
void launch_points_real(int nt, const double* tc, const double* tblur, int ns, const double4* s4s,
                        const int* sperm, const double* sc, const double* sblur,
                        const int* box_start, const PointsReal& g, double* pot, double* grad,
                        cudaStream_t st);
// x[0..n) = v.
void launch_fill(double* x, int n, double v, cudaStream_t st);
// dst(3, n) += scale_i src(3, n) (scale NULL: 1).
void launch_add_scaled3(int n, const double* scale, const double* src, double* dst,
                        cudaStream_t st);

int mesh_configure_kernels();
// Dense FP64 tensor-core (DMMA m8n8k4) rate of this GPU in TFLOP/s, timed on `st`.
int measure_dmma_peak(cudaStream_t st, double* tflops);
// EWG_ERR_GRID_TOO_LARGE when one line of an axis does not fit a pass CTA's shared
// memory (a guard: every length up to kMaxFftLength fits in both precisions).
int mesh_check_lengths(const MeshGeom& g, bool mixed);
int stencil_configure_kernels();

}  // namespace ewg
