// ewg_static.cu -- the direct Ewald engine without any allocation.
//
// ewg_direct_potential_force_static computes what ewg_direct_potential_force
// computes, on arrays the caller already holds in device memory, and takes all
// of its working memory from one fixed array in device global memory
// (g_static_scratch below).  It never calls cudaMalloc, cudaFree or any other
// allocating routine, host or device.
//
// Why: some host codes cannot allocate device memory once a run is under way,
// for example a program that hands all device memory to its own pool allocator
// at start-up, or one that must not risk an allocation failing or stalling in
// the middle of a molecular-dynamics or SCC loop.  Those callers can still
// evaluate the direct engine (the validation engine the reference adapter
// selects with DFTB_EWALD_DIRECT=1), within the size limit below.
//
// Limits and sharing.  The array is kStaticScratchBytes (16 MiB) on every GPU
// that loads the library, held until the process exits.  Atoms, cell-list
// boxes and Fourier modes are carved from it; a configuration that does not fit
// is rejected with EWG_ERR_SCRATCH_LIMIT before any kernel runs (about 100,000
// atoms with few modes, fewer when the mode box is large).  Every call shares
// the array: calls that overlap on the GPU (two streams, two host threads)
// race and give wrong results.  The array keeps the last call's contents;
// everything that must start at zero is cleared on the call's stream.
//
// Set-up: the device address of the array is looked up once per device, with
// that device current, on the first call made on it (cudaGetSymbolAddress);
// later calls reuse it.  Make that first call on each device before any stream
// capture begins.  With CUDA's lazy module loading (the default since CUDA
// 12.2) the 16 MiB array is only reserved on a device when this file's module
// first loads there, which is that same first call.  A program that hands all
// device memory to its own pool at start-up must therefore make one call on
// each device (any small system will do) before its pool takes the memory;
// otherwise the first call can fail with EWG_ERR_OUT_OF_MEMORY.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "ewg_kernels.h"

namespace ewg {
namespace {

constexpr size_t kStaticScratchBytes = size_t(16) << 20;
constexpr int kMaxDevices = 64;
constexpr int kSumBlocks = 148;

__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_scratch_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array for the current device.
int scratch_address(unsigned char** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return EWG_ERR_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      // Under lazy module loading this lookup is what loads the module and
      // reserves the array; with the device memory already taken it fails here.
      return e == cudaErrorMemoryAllocation ? EWG_ERR_OUT_OF_MEMORY : EWG_ERR_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_ptr[dev];
  return EWG_OK;
}

// Bump carving of the scratch array, 256-byte aligned pieces.
struct Carve {
  unsigned char* base;
  size_t off = 0;
  template <class T>
  T* take(size_t count) {
    off = (off + 255) & ~size_t(255);
    T* p = reinterpret_cast<T*>(base + off);
    off += count * sizeof(T);
    return p;
  }
  bool fits() const { return off <= kStaticScratchBytes; }
};

// Mode box of the direct Fourier sum (direct/ewald_direct_3d.f90:131-174):
// (mx, my, mz) in [-nm, nm]^3 in the reference's loop order, mz fastest.
struct ModeBox {
  int nm[3];
  double rec[3][3];
  double kc2, volume, alpha;
};

__device__ __forceinline__ bool mode_vector(const ModeBox& b, int v, double* k, double* k2) {
  const int sz = 2 * b.nm[2] + 1, sy = 2 * b.nm[1] + 1;
  const int mz = v % sz - b.nm[2];
  const int my = (v / sz) % sy - b.nm[1];
  const int mx = v / (sz * sy) - b.nm[0];
  for (int d = 0; d < 3; ++d)
    k[d] = (mx * b.rec[0][d] + my * b.rec[1][d] + mz * b.rec[2][d]) * 2.0 * 3.14159265358979323846;
  *k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
  return !(*k2 < 1.0e-24 || *k2 > b.kc2);
}

// Per mode: Cartesian vector, weight, and structure factor (one CTA per mode).
__global__ void __launch_bounds__(256) k_modes_box(const double* __restrict__ x,
                                                   const double* __restrict__ q, int n, ModeBox b,
                                                   double* __restrict__ modes /* 6 per mode */) {
  __shared__ double sh[2][8];
  const int v = blockIdx.x;
  double k[3], k2;
  const bool in = mode_vector(b, v, k, &k2);
  double sr = 0.0, si = 0.0;
  if (in) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      double sn, cs;
      sincos(k[0] * x[3 * i] + k[1] * x[3 * i + 1] + k[2] * x[3 * i + 2], &sn, &cs);
      sr += q[i] * cs;
      si += q[i] * sn;
    }
    for (int off = 16; off > 0; off >>= 1) {
      sr += __shfl_down_sync(0xffffffffu, sr, off);
      si += __shfl_down_sync(0xffffffffu, si, off);
    }
    if ((threadIdx.x & 31) == 0) {
      sh[0][threadIdx.x >> 5] = sr;
      sh[1][threadIdx.x >> 5] = si;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double* m = modes + 6 * static_cast<size_t>(v);
    double a = 0.0, c = 0.0, w = 0.0;
    if (in) {
      for (int j = 0; j < 8; ++j) {
        a += sh[0][j];
        c += sh[1][j];
      }
      w = 4.0 * 3.14159265358979323846 / b.volume * exp(-k2 / (4.0 * b.alpha * b.alpha)) / k2;
    }
    m[0] = k[0];
    m[1] = k[1];
    m[2] = k[2];
    m[3] = w;
    m[4] = a;
    m[5] = c;
  }
}

// Fourier part per atom over the whole box in the reference's order, skipping
// modes outside the sphere; then the self term (ewald_self.f90:12-19).
__global__ void __launch_bounds__(256) k_kspace_self(const double* __restrict__ x,
                                                     const double* __restrict__ q, int n,
                                                     const double* __restrict__ modes, int nmodes,
                                                     double self_coef, double* __restrict__ pot,
                                                     double* __restrict__ force) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2];
  double p = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
  for (int v = 0; v < nmodes; ++v) {
    const double* m = modes + 6 * static_cast<size_t>(v);
    const double w = m[3];
    if (w == 0.0) continue;
    double sn, cs;
    sincos(m[0] * xi + m[1] * yi + m[2] * zi, &sn, &cs);
    const double lr = m[4] * cs + m[5] * sn;
    const double li = m[5] * cs - m[4] * sn;
    p += w * lr;
    const double ff = w * li;
    fx -= ff * m[0];
    fy -= ff * m[1];
    fz -= ff * m[2];
  }
  pot[i] = (pot[i] + p) + self_coef * q[i];
  force[3 * i] += q[i] * fx;
  force[3 * i + 1] += q[i] * fy;
  force[3 * i + 2] += q[i] * fz;
}

}  // namespace
}  // namespace ewg

using namespace ewg;

extern "C" int ewg_direct_potential_force_static(int n, const double* coords_device,
                                                 const double* charges_device,
                                                 const double* lat_rows, double tol,
                                                 double* pot_device, double* force_device,
                                                 const double* alpha_in, const double* r_cut_in,
                                                 const double* k_cut_in, void* stream) {
  if (n <= 0) return EWG_ERR_NPARTICLE;
  if (!coords_device || !charges_device || !lat_rows || !pot_device) return EWG_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  Carve cv{base};
  double* partial = cv.take<double>(3 * kSumBlocks);
  double* sums = cv.take<double>(4);
  int* err = cv.take<int>(1);

  // check_configuration (common/ewald_validation.f90:26-48) on the device charges.
  launch_charge_sums(charges_device, n, partial, sums, st);
  double h[3];
  cudaError_t e = cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? EWG_ERR_OUT_OF_MEMORY : EWG_ERR_CUDA;
  if ((rc = check_sums(n, h[0], h[1]))) return rc;
  Cell cell;
  if ((rc = cell_from_rows(lat_rows, cell))) return rc;
  if (!(tol > 0.0 && tol < 1.0)) return EWG_ERR_TOL;

  // Splitting and cutoffs (direct/ewald_direct_3d.f90:105-120).
  const double alpha = alpha_in ? *alpha_in : balanced_splitting(cell, tol);
  if (!(alpha > 0.0)) return EWG_ERR_ALPHA;
  double r_cut = 0.0, k_cut = 0.0;
  if (!(r_cut_in && k_cut_in)) {
    r_cut = std::sqrt(-std::log(tol)) / alpha;
    k_cut = 2.0 * alpha * std::sqrt(-std::log(tol));
  }
  if (r_cut_in) r_cut = *r_cut_in;
  if (k_cut_in) k_cut = *k_cut_in;
  if (!(r_cut > 0.0) || !(k_cut > 0.0)) return EWG_ERR_CUTOFF;

  // Cell list for the real-space image sum: boxes at least r_cut wide, capped
  // at 4 per atom (wider boxes stay correct).
  RealGeom rg;
  for (int d = 0; d < 3; ++d) rg.nb[d] = std::max(1, std::min(box_count(r_cut, cell.recLen[d]), 1 << 10));
  const long cap = std::max<long>(64, 4L * n);
  while (static_cast<long>(rg.nb[0]) * rg.nb[1] * rg.nb[2] > cap) {
    int d = 0;
    if (rg.nb[1] > rg.nb[d]) d = 1;
    if (rg.nb[2] > rg.nb[d]) d = 2;
    rg.nb[d] = std::max(1, rg.nb[d] / 2);
  }
  for (int d = 0; d < 3; ++d) {
    rg.R[d] = std::max(1, static_cast<int>(std::ceil(r_cut * cell.recLen[d] * rg.nb[d])));
    for (int f = 0; f < 3; ++f) {
      rg.lat[d][f] = cell.lat[d][f];
      rg.rec[d][f] = cell.rec[d][f];
    }
  }
  set_scan_mode(rg);
  const int nboxes = rg.nb[0] * rg.nb[1] * rg.nb[2];
  ModeBox mb;
  long nmodes = 1;
  for (int d = 0; d < 3; ++d) {
    mb.nm[d] = static_cast<int>(std::ceil(k_cut * cell.latLen[d] / (2.0 * kPi))) + 1;
    nmodes *= 2L * mb.nm[d] + 1;
    for (int f = 0; f < 3; ++f) mb.rec[d][f] = cell.rec[d][f];
  }
  mb.kc2 = k_cut * k_cut;
  mb.volume = cell.volume;
  mb.alpha = alpha;

  // Everything else from the scratch array, or a clear refusal.
  if (nmodes > (1L << 24)) return EWG_ERR_SCRATCH_LIMIT;
  double4* s4 = cv.take<double4>(n);
  double4* s4s = cv.take<double4>(n);
  float4* x32s = cv.take<float4>(n);
  int* boxkey = cv.take<int>(n);
  int* counts = cv.take<int>(nboxes);
  int* cursor = cv.take<int>(nboxes);
  int* starts = cv.take<int>(nboxes + 1);
  int* tmp = cv.take<int>(n);
  int* perm = cv.take<int>(n);
  double* fbuf = force_device ? force_device : cv.take<double>(3 * static_cast<size_t>(n));
  double* modes = cv.take<double>(6 * static_cast<size_t>(nmodes));
  if (!cv.fits()) return EWG_ERR_SCRATCH_LIMIT;

  cudaMemsetAsync(err, 0, sizeof(int), st);
  launch_atom_prep(coords_device, 3, 1, charges_device, n, cell, rg.nb, nullptr, s4, boxkey,
                   nullptr, nullptr, st);
  launch_bucket_sort(boxkey, n, nboxes, counts, cursor, starts, tmp, perm, st);
  launch_permute_box(s4, perm, n, cell.lat, s4s, x32s, st);
  launch_real_space(s4s, x32s, perm, starts, n, rg, alpha, r_cut, 0, pot_device, fbuf, err, st);
  k_modes_box<<<static_cast<unsigned>(nmodes), 256, 0, st>>>(coords_device, charges_device, n, mb,
                                                             modes);
  k_kspace_self<<<(n + 255) / 256, 256, 0, st>>>(coords_device, charges_device, n, modes,
                                                  static_cast<int>(nmodes),
                                                  -2.0 * alpha / std::sqrt(kPi), pot_device, fbuf);
  g_launches += 2;
  int herr = 0;
  e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? EWG_ERR_OUT_OF_MEMORY : EWG_ERR_CUDA;
  return herr ? EWG_ERR_COINCIDENT : EWG_OK;
}
