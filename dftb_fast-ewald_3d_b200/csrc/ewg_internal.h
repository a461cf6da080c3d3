// ewg_internal.h -- declarations shared by the host chain, the kernels and the
// C ABI of the B200 Ewald operator.  Not installed; include/ewald_b200.h is the
// public interface.
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/ewald_b200.h"

namespace ewg {

// ---------------------------------------------------------------------------
// Host side: geometry and the reference's parameter chain (ewg_chain.cpp)
// ---------------------------------------------------------------------------

// TCell3d (common/ewald_geometry.f90:22-44).  lat[i][d] is lattice vector a_i,
// rec[i][d] the dual vector b_i with b_i . a_j = delta_ij (no factor 2 pi).
struct Cell {
  double lat[3][3];
  double rec[3][3];
  double volume;
  double latLen[3];
  double recLen[3];
};

// cell_metrics_3d (common/ewald_geometry.f90:65-93) from the Fortran rows layout.
int cell_from_rows(const double* lat_rows, Cell& cell);
// The same geometry from DFTB+'s column layout (coulomb.F90 latVecs_(:, i) = a_i).
int cell_from_cols(const double* lat_cols, Cell& cell);

// check_configuration (common/ewald_validation.f90:26-48) on host charges;
// also returns sum q^2 for the parameter chain.
int check_charges(int n, const double* q, double* q2sum, double* qsum = nullptr);
// The same test on the three sums (sum q, sum |q|, sum q^2).
int check_sums(int n, double sum_q, double sum_abs_q);

// choose_parameters (fft/ewald_fft_3d_parameters.f90:52-142).
int choose_parameters(const Cell& cell, double q2sum, int n, double tol, const ewg_overrides* ov,
                      ewg_params& p);
// grid_memory_gigabytes (fft/ewald_fft_3d_parameters.f90:177-229).
double grid_memory_gigabytes(const ewg_params& p);
int next_fast_length(int n);      // nfft/fft_backend.f90:73-91
double window_shape(int m);       // nfft/nfft.f90:82-92
int box_count(double r_cut, double recLen);  // common/ewald_cell_list.f90:56-73

// Balanced splitting of the direct engine (direct/ewald_direct_3d.f90:319-347).
double balanced_splitting(const Cell& cell, double tol);

// Stock DFTB+ setup used by invRStress (coulomb.F90:575-620, :2097-2308).
struct StockSetup {
  double alpha, max_r, max_g;
  std::vector<double> g;  // Cartesian half-space reciprocal vectors, 3 per point
};
int stock_setup(const Cell& cell, double tol_ewald, double alpha_in, StockSetup& out);

constexpr double kPi = 3.14159265358979323846;
constexpr int kOversampling = 2;  // nfft/nfft.f90:43

// ---------------------------------------------------------------------------
// Device side
// ---------------------------------------------------------------------------

constexpr int kMaxFftLength = 4096;
constexpr int kMaxStages = 16;

// One FFT length: its radix schedule and a device twiddle table
// tw[k] = exp(-2 pi i k / n), k in [0, n).
struct FftPlan {
  int n = 0;
  int nstages = 0;
  int radix[kMaxStages] = {0};
  const double* tw64 = nullptr;  // interleaved complex, device
  const float* tw32 = nullptr;   // interleaved complex, device
};

// Everything the mesh kernels need about one evaluation.
struct MeshGeom {
  int n[3];        // fine grid = 2 * modes
  int M[3];        // retained modes
  int K1, K2, K3;  // compact spectrum extents: M1/2+1, M2+1, M3+1
  int m;           // window half-width
  int W;           // 2m+1
  double b;        // window shape
  double pref;     // 1/sqrt(pi b)
  double rec[3][3];
  double volume, alpha;
};

struct RealGeom {
  int nb[3];       // boxes per axis
  int R[3];        // neighbour box range per axis
  int flat;        // 1: the neighbourhood has at most 32 rows (dy, dz) and each
                   // row is at most two contiguous runs of boxes (see set_scan_mode)
  double lat[3][3];
  double rec[3][3];
  double rl[3];    // |rec_d|: fractional extent per Bohr normal to the planes s_d = const
  double h[3];     // 1 / rl[d]: spacing of the planes s_d = 0 and s_d = 1
  double inb[3];   // 1 / nb[d]
  int ortho;       // 1: the three plane normals are mutually orthogonal
  int rowmul;      // ceil(2^16 / (2 R_y + 1)): row / (2 R_y + 1) as (row * rowmul) >> 16, exact for rows < 32
};

// The flat candidate scan needs every x row of 2R+1 boxes to split into at
// most two runs (nb_x >= 2R_x + 1) and at most 32 rows.  Also fills rl and
// ortho, which the scan uses to skip rows and trim runs beyond the cutoff.
inline void set_scan_mode(RealGeom& g) {
  const int rows = (2 * g.R[1] + 1) * (2 * g.R[2] + 1);
  g.flat = (g.nb[0] >= 2 * g.R[0] + 1 && rows <= 32) ? 1 : 0;
  for (int d = 0; d < 3; ++d) {
    g.rl[d] = std::sqrt(g.rec[d][0] * g.rec[d][0] + g.rec[d][1] * g.rec[d][1] +
                        g.rec[d][2] * g.rec[d][2]);
    g.h[d] = 1.0 / g.rl[d];
    g.inb[d] = 1.0 / g.nb[d];
  }
  g.rowmul = (65536 + 2 * g.R[1]) / (2 * g.R[1] + 1);
  g.ortho = 1;
  for (int d = 0; d < 3; ++d)
    for (int e = d + 1; e < 3; ++e) {
      const double dot = g.rec[d][0] * g.rec[e][0] + g.rec[d][1] * g.rec[e][1] +
                         g.rec[d][2] * g.rec[e][2];
      if (std::fabs(dot) > 1e-12 * g.rl[d] * g.rl[e]) g.ortho = 0;
    }
}

}  // namespace ewg
