/*
 * ewald_oracle.h -- TEST INFRASTRUCTURE, NOT THE PRODUCT.
 *
 * CPU restatement (C++17 + OpenMP) of the reference's fast 3D Ewald library
 * (src/dftbp/extlibs/fftewald, all modules) and of DFTB+'s stock Ewald stress
 * (src/dftbp/dftb/coulomb.F90 invRStress and its setup).  It is the checker for
 * the CUDA library: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.
 *
 * Parity status: parity unpinned.  The reference ships no test, golden vector or
 * known-answer case for this path (its only periodic Coulomb unit test has its
 * assertions commented out), and the reference cannot be built in this image
 * (no Fortran compiler, no FFTW).  The restatement is cross-checked instead
 * against an independent numpy implementation, the rock-salt Madelung constant,
 * the direct O(N^2) engine and finite differences (tests/).
 *
 * Array conventions follow the reference library:
 *   positions  : Fortran positions(N,3), column-major: positions[i + N*d]
 *   latVecs    : Fortran latVecs(3,3), one lattice vector per ROW,
 *                column-major storage: a_i component d at lat[i + 3*d]
 *   force      : Fortran force(3,N): force[d + 3*i]
 * The stock-stress entry takes DFTB+'s own conventions (coords(3,N), latVecs
 * with one vector per COLUMN).
 */
#ifndef EWALD_ORACLE_H
#define EWALD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes; the numbering matches include/ewald_b200.h. */
enum {
  EWO_OK = 0,
  EWO_ERR_NPARTICLE = 1,
  EWO_ERR_ARG = 2,
  EWO_ERR_NOT_NEUTRAL = 3,
  EWO_ERR_TOL = 4,
  EWO_ERR_VOLUME = 5,
  EWO_ERR_ALPHA = 6,
  EWO_ERR_COINCIDENT = 7,
  EWO_ERR_CUTOFF = 8,
  EWO_ERR_ALPHA_SEARCH = 9,
  EWO_ERR_LATTICE_SEARCH = 10
};

/* Optional arguments of ewald_potential_force (fft/ewald_fft_3d.f90:36-77). */
typedef struct {
  int has_alpha, has_r_cut, has_k_cut, has_n_modes, has_window_cutoff;
  double alpha, r_cut, k_cut;
  int n_modes, window_cutoff;
} ewo_overrides;

/* TEwaldParameters3d (fft/ewald_fft_3d_parameters.f90:24-42). */
typedef struct {
  double alpha, r_cut, k_cut;
  int window_cutoff;
  int n_modes[3];
} ewo_params;

int ewo_set_threads(int n);

int ewo_fft_potential_force(int n, const double* positions, const double* charges,
                            const double* lat, double tol, double* pot, double* force,
                            const ewo_overrides* ov);
int ewo_fft_parameters(int n, const double* charges, const double* lat, double tol,
                       const ewo_overrides* ov, ewo_params* out);
int ewo_fft_grid_memory(int n, const double* charges, const double* lat, double tol,
                        const ewo_overrides* ov, double* gigabytes);
int ewo_direct_potential_force(int n, const double* positions, const double* charges,
                               const double* lat, double tol, double* pot, double* force,
                               const double* alpha_in, const double* r_cut_in,
                               const double* k_cut_in);
/* Wall-clock seconds of the last ewo_fft_potential_force: real space, spread,
 * FFTs, gathers, other (out: 5 doubles). */
int ewo_stage_seconds(double* out);
int ewo_real_space(int n, const double* positions, const double* charges, const double* lat,
                   double alpha, double r_cut, double* pot, double* force, int* used_cell_list);

/* Stock DFTB+ electrostatic stress: coulomb.F90 updateLatVecs (:575-620) followed
 * by invRStress (:2777-2863).  coords(3,N), latVecs with one vector per column.
 * alpha <= 0 selects getOptimalAlphaEwald.  stress_out receives invRStress's
 * tensor (column-major 3x3); TCoulomb%addStress subtracts half of it. */
int ewo_stock_stress(int n, const double* coords, const double* dq, const double* lat_cols,
                     double tol_ewald, double alpha, double* stress_out, double* alpha_out,
                     double* max_r_out, double* max_g_out, int* n_g_out);

/* Source -> target potentials and gradients of TCoulomb (coulomb.F90:3122-3248),
 * stock Ewald sum with updateLatVecs's setup.  Coordinates (3,n) atom-major,
 * latVecs one vector per column, alpha <= 0 selects getOptimalAlphaEwald.
 * blur (per source) and eps_soften may be NULL.  Gradients (3,n). */
int ewo_potential_at(int nt, const double* tcoords, int ns, const double* scoords,
                     const double* scharges, const double* blur, const double* eps_soften,
                     const double* lat_cols, double tol_ewald, double alpha, double* pot);
int ewo_potential_gradient_at(int nt, const double* tcoords, int ns, const double* scoords,
                              const double* scharges, const double* blur, const double* lat_cols,
                              double tol_ewald, double alpha, double* grad);
int ewo_external_pot_grad(int na, const double* acoords, int ne, const double* ecoords,
                          const double* acharges, const double* echarges, int ham_deriv,
                          const double* eblur, const double* lat_cols, double tol_ewald,
                          double alpha, double* agrad, double* egrad);

/* XLBOMD gradients of the shadow energy with input and output charges,
 * addInvRPrimeXlbomdPeriodic (coulomb.F90:1823-1894), stock Ewald; adds to
 * deriv(3,n). */
int ewo_xlbomd_gradients(int n, const double* coords, const double* dq_in, const double* dq_out,
                         const double* lat_cols, double tol_ewald, double alpha, double* deriv);

/* Building blocks, exposed for the cross-checks. */
int ewo_fft3d(int n1, int n2, int n3, double* data /* complex interleaved */, int isign);
int ewo_adjoint_nfft(int n, const double* t1, const double* t2, const double* t3,
                     const double* q, int M1, int M2, int M3, int m, double* shat);
int ewo_forward_nfft(int n, const double* t1, const double* t2, const double* t3, int M1, int M2,
                     int M3, int m, const double* fhat, double* f);
int ewo_next_fast_length(int n);
double ewo_lambert_w0(double x);

#ifdef __cplusplus
}
#endif
#endif
