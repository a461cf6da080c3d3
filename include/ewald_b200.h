/*
 * ewald_b200.h -- C ABI of the B200 (sm_100a) 3D-periodic Ewald operator.
 *
 * This library replaces the engine behind DFTB+'s TCoulomb call surface for
 * three-dimensionally periodic, charge-neutral SCC calculations: the real-space
 * erfc pair sum over a linked-cell list, the Gaussian-window NFFT reciprocal
 * sum (spread, FFT, influence weights, gather) and the stock electrostatic
 * stress.  Every function returns an int status (EWG_OK == 0); see
 * ewg_status_string().  All pointers are host memory unless a name ends in
 * _device.  Outputs are overwritten, never accumulated into.
 *
 * Array conventions (atomic units: Bohr, e, Hartree):
 *   positions(N,3)  Fortran column-major, as the reference library takes them:
 *                   atom i component d at positions[i + N*d].
 *   coords(3,N)     DFTB+'s own layout: atom i component d at coords[d + 3*i].
 *   lat_rows(3,3)   Fortran latVecs with one lattice vector per ROW,
 *                   column-major: a_i component d at lat_rows[i + 3*d].
 *   lat_cols(3,3)   DFTB+'s latVecs with one lattice vector per COLUMN:
 *                   a_i component d at lat_cols[d + 3*i].
 *   force(3,N)      physical force -dU/dx, atom i component d at force[d + 3*i].
 *
 * Threading: one context per host thread; a context is not re-entrant.  Each
 * context owns one CUDA stream and its device buffers; every call completes on
 * the GPU before it returns.
 */
#ifndef EWALD_B200_H
#define EWALD_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
/* Each replaces an `error stop` of the reference (paths relative to the
 * reference project); a Fortran adapter maps non-zero codes back to
 * `error stop ewg_status_string(rc)`. */
enum {
  EWG_OK = 0,
  EWG_ERR_NPARTICLE = 1,    /* common/ewald_validation.f90:34  nParticle <= 0            */
  EWG_ERR_ARG = 2,          /* NULL pointer, bad precision mode, shape mismatch            */
  EWG_ERR_NOT_NEUTRAL = 3,  /* common/ewald_validation.f90:43-46  |sum q| > 1e-8 sum|q|   */
  EWG_ERR_TOL = 4,          /* fft/ewald_fft_3d.f90:97-98  tol outside (0,1)              */
  EWG_ERR_VOLUME = 5,       /* common/ewald_geometry.f90:78  cell volume <= 1e-18         */
  EWG_ERR_ALPHA = 6,        /* fft/ewald_fft_3d_parameters.f90:121  alpha <= 0            */
  EWG_ERR_COINCIDENT = 7,   /* fft/ewald_fft_3d_real.f90:159-160  r^2 < 1e-24             */
  EWG_ERR_CUTOFF = 8,       /* direct/ewald_direct_3d.f90:117-118  cutoffs <= 0           */
  EWG_ERR_ALPHA_SEARCH = 9, /* dftb/coulomb.F90:2172-2177  getOptimalAlphaEwald failed    */
  EWG_ERR_LATTICE_SEARCH = 10, /* dftb/coulomb.F90:2239-2243, :2304-2308 getMaxG/REwald   */
  EWG_ERR_OUT_OF_MEMORY = 11,
  EWG_ERR_CUDA = 12,
  EWG_ERR_DEVICE_TIMEOUT = 13,
  EWG_ERR_GRID_TOO_LARGE = 14, /* an FFT length beyond the kernels' limit (4096 per axis)  */
  EWG_ERR_NO_DEVICE = 15,
  EWG_ERR_STATE = 16,       /* call order: dftb/coulomb.F90 @:ASSERT(coordsUpdated_) etc. */
  EWG_ERR_SCRATCH_LIMIT = 17 /* configuration too large for the fixed scratch of
                                ewg_direct_potential_force_static                   */
};

/* ---- precision forms ---------------------------------------------------- */
enum {
  EWG_PRECISION_FP64 = 0,  /* plain form: FP64 throughout, parity with the reference  */
  EWG_PRECISION_MIXED = 1  /* FP32 window weights, grids, FFT and pair terms; the
                              stencil contractions on the FP64 tensor cores (or FP32
                              CUDA cores, ewg_kernel_shape.stencil); FP64 accumulation,
                              self term, reductions and lattice setup                 */
};

/* ---- force differentiation schemes --------------------------------------- */
enum {
  EWG_FORCE_IK = 0, /* the reference's scheme: the potential spectrum times i k per
                       Cartesian component, four inverse transforms and gathers
                       (fft/ewald_fft_3d_fourier.f90:130-151)                    */
  EWG_FORCE_AD = 1  /* analytic differentiation of the window: one inverse
                       transform; the gather applies the window and its
                       derivative along each fractional axis                     */
};

/* ---- engines of the potentials at arbitrary points ----------------------- */
enum {
  EWG_POINTS_AUTO = 0,  /* mesh from 2^20 (target, source) pairs on, stock below    */
  EWG_POINTS_STOCK = 1, /* the reference's stock pair sum, O(N_t N_s) (default for
                           small inputs)                                           */
  EWG_POINTS_MESH = 2   /* NFFT reciprocal sum plus a cell-list real-space sum,
                           O(N_t + N_s)                                            */
};

/* Optional arguments of ewald_potential_force (fft/ewald_fft_3d.f90:36-77):
 * alpha_in, r_cut_in, k_cut_in, nModes_in, windowCutoff_in.  A member counts
 * only when its has_ flag is non-zero. */
typedef struct {
  int has_alpha, has_r_cut, has_k_cut, has_n_modes, has_window_cutoff;
  double alpha, r_cut, k_cut;
  int n_modes, window_cutoff;
} ewg_overrides;

/* TEwaldParameters3d (fft/ewald_fft_3d_parameters.f90:24-42). */
typedef struct {
  double alpha, r_cut, k_cut;
  int window_cutoff;
  int n_modes[3];
} ewg_params;

typedef struct ewg_context ewg_context;

/* ---- context ------------------------------------------------------------ */
int ewg_create(ewg_context** ctx, int device, int precision);
int ewg_destroy(ewg_context* ctx);
const char* ewg_status_string(int status);
/* Run the context's work on the caller's CUDA stream (a cudaStream_t passed as
 * void*); NULL returns to the context's own stream.  Calls still complete on
 * the GPU before they return. */
int ewg_set_stream(ewg_context* ctx, void* stream);
/* CUDA graphs (on by default): an evaluation whose launch sequence -- sizes,
 * device pointers, parameters, cell, stream -- repeats is recorded as a CUDA
 * graph on its second call and replayed from the third, one graph launch in
 * place of some twenty kernel launches.  Off with on = 0 (recorded graphs are
 * released).  Not used while stage profiling is on. */
int ewg_set_graphs(ewg_context* ctx, int on);
/* Number of this library's kernels launched by the context so far. */
long long ewg_kernel_launches(const ewg_context* ctx);
/* Charged cells (on != 0): the fast path then accepts a net charge Q, with the
 * uniform neutralising background the stock Ewald engine implies (its pair
 * function carries -pi/(V alpha^2) per unit charge, dftb/coulomb.F90:2338):
 * every potential gains -pi Q/(V alpha^2) with the evaluation's alpha, forces
 * are unchanged, and the stresses of ewg_potential_force_stress / ewg_stress_fast
 * include the background energy -pi Q^2/(2 V alpha^2).  The reference's fast
 * path refuses charged cells (common/ewald_validation.f90:43-46); this mode
 * has no counterpart there (fft3d_readme.md:31).  Off by default. */
int ewg_set_background(ewg_context* ctx, int on);
/* Force differentiation scheme of the context's force evaluations
 * (EWG_FORCE_IK or EWG_FORCE_AD).  Default: IK, the reference's own scheme,
 * in both precision forms.  AD computes the
 * reciprocal force as -q sum_d b_d sum_l g_l dW/ds_d, with g the potential grid
 * and W the product of the three Gaussian windows; it spends one inverse
 * transform where IK spends four.  Both converge to the same Ewald force; at
 * the reference's parameters for tol = 1e-10 they differ by about 1e-12
 * relative.  Potentials, energies and stresses do not depend on the scheme.
 * In FP32 (the mixed form) ad is less robust: the derivative sums cancel, and
 * in strongly anisotropic cells its error can exceed the i k form's by an
 * order of magnitude; ewg_tune measures both and picks.
 * No counterpart in the reference. */
int ewg_set_force_scheme(ewg_context* ctx, int scheme);
/* Engine of ewg_potential_at, ewg_potential_gradient_at and
 * ewg_external_pot_grad (EWG_POINTS_AUTO, _STOCK or _MESH; default AUTO).
 * STOCK evaluates the reference's pair function ewald (dftb/coulomb.F90:2311-2343)
 * for every (target, source) pair with DFTB+'s own splitting: O(N_t N_s) with a
 * real-space sum over every cell translation.  MESH computes the same periodic
 * sum, which does not depend on the splitting, at cost O(N_t + N_s): alpha,
 * cutoffs, window and grid from the fast path's parameter chain for the
 * sources at tol_ewald, the Fourier part through the NFFT (sources spread,
 * targets gathered, gradients by window differentiation), the real-space part
 * (with each source's Gaussian blur) over a cell list within the chain's
 * cutoff widened to the widest blur, all in FP64.  The two agree to the
 * truncation of either method at tol_ewald (about 1e-9 relative at 1e-10).
 * The alpha argument of those calls then plays no part.  A softening length
 * is defined on the stock splitting (the reference softens only its
 * real-space part), so a call with eps_soften != 0 always takes the stock sum.
 * The reference's own next step for these routines is such an operator
 * (fft3d_readme.md:36). */
int ewg_set_point_engine(ewg_context* ctx, int engine);
/* Parameters the last evaluation on this context used. */
int ewg_last_params(const ewg_context* ctx, ewg_params* out);
/* Measured dense FP64 tensor-core rate of the context's GPU (DMMA m8n8k4 on
 * register operands, all SMs, CUDA-event timed), in TFLOP/s: the roofline
 * denominator of the FP64 spread and gather.  Diagnostic; no counterpart in
 * the reference. */
int ewg_fp64_mma_peak(ewg_context* ctx, double* tflops);

/* ---- per-stage device timing ------------------------------------------- */
/* With profiling on, every evaluation records CUDA events on the context's
 * stream around each stage (atom preparation and sorting, real-space sum,
 * window weights, spread, the five FFT passes, gather) and accumulates their
 * device durations.  Stage names: ewg_stage_name(i), 0 <= i < ewg_stage_count(). */
int ewg_set_profiling(ewg_context* ctx, int on);
int ewg_stage_count(void);
const char* ewg_stage_name(int stage);
/* Accumulated milliseconds and launch counts per stage since the last reset. */
int ewg_stage_times(const ewg_context* ctx, double* ms, long long* launches, int n);
int ewg_reset_stage_times(ewg_context* ctx);

/* ---- library surface: fft/ewald_fft_3d.f90 ------------------------------ */

/* ewald_potential_force (fft/ewald_fft_3d.f90:36-134).  force may be NULL:
 * potential-only evaluation with one forward transform instead of four.
 * ov may be NULL (no overrides).  When ov fixes alpha and k_cut and the
 * background convention is off, the parameters do not depend on the charges:
 * the evaluation is queued first and the charges are checked while it runs
 * (EWG_ERR_NOT_NEUTRAL is then reported after the cell and tolerance checks).
 * On every error return pot and force are left as they were. */
int ewg_potential_force(ewg_context* ctx, int n, const double* positions, const double* charges,
                        const double* lat_rows, double tol, double* pot, double* force,
                        const ewg_overrides* ov);

/* ewald_potential_force plus the stress of the same evaluation, from the same
 * NFFT spectrum: sigma (3 x 3, column-major, symmetric) = (2/V) dE/d(strain)
 * with E = 1/2 sum_i q_i pot_i, the quantity invRStress returns
 * (dftb/coulomb.F90:2777-2863; the caller does stress -= 0.5 sigma).  Real
 * space: the virial of the erfc pair term over the evaluation's own pairs;
 * reciprocal space: sum_k 1/2 w(k) |G(k)|^2 (2 k k (1/(4 alpha^2) + 1/k^2) - 1)
 * over the NFFT modes.  It uses the fast path's alpha and cutoffs, not the stock
 * engine's.  The reference lists this as its next step for the fast path
 * (fft3d_readme.md:30); it has no implementation to compare with. */
int ewg_potential_force_stress(ewg_context* ctx, int n, const double* positions,
                               const double* charges, const double* lat_rows, double tol,
                               double* pot, double* force, double* sigma,
                               const ewg_overrides* ov);

/* Parameter autotuner for the context's precision form (the mixed form in
 * practice).  On the caller's configuration it evaluates candidates -- both
 * force schemes, with the reference chain at tol = target/10, /5, /3, the
 * real-space cutoff scaled by 0.7, 0.85, 1, 1.15, 1.3 or 1.5 (alpha, k_cut and
 * the modes following from it) and window half-widths 5..9 -- against an FP64 i k
 * evaluation at the reference's parameters for tol = 1e-10, times those whose
 * RMS relative force error is at most target/2 and RMS relative potential
 * error at most target, and returns the fastest: its parameters as overrides
 * (alpha, r_cut, k_cut, window_cutoff; any tol in (0,1) may accompany them)
 * and its force scheme in *scheme (may be NULL; apply it with
 * ewg_set_force_scheme).  If no candidate meets the bar, the most accurate one
 * is returned.  report (optional, 4 doubles): its force and potential RMS
 * errors, its device milliseconds per force evaluation, and the number of
 * candidates evaluated.  Results are cached in the context per (atoms, form,
 * lattice, target); the context's force scheme is left as it was.  The
 * winner's kernel shapes are then tuned as by ewg_tune_kernels, so later
 * evaluations with the returned overrides run them.
 * No counterpart in the reference. */
int ewg_tune(ewg_context* ctx, int n, const double* positions, const double* charges,
             const double* lat_rows, double target, ewg_overrides* out, int* scheme,
             double* report);

/* Kernel shapes of an evaluation.  A field left 0 takes the library's default.
 * Results do not depend on gather_warps or fft_lines (bitwise); box_div,
 * fft_sched and stencil change the order or the precision of the sums, so
 * results move by rounding only.
 * No counterpart in the reference (its kernels are fixed CPU loops). */
typedef struct {
  int box_div;      /* real-space cell list: boxes per reference box width
                       (box_count_3d, common/ewald_cell_list.f90:56-73) along
                       each axis, 1, 2 or 3 (default 2: 5 x 5 x 5 neighbourhoods) */
  int fft_lines;    /* most FFT lines per CTA: 1, 2, 4 or 8 (default: the most
                       whose buffers fit the CTA's shared-memory budget) */
  int fft_sched;    /* FFT radix schedule: 1 odd radices, then radix 8 (default);
                       2 odd radices, then radix 4 in place of 8 */
  int gather_warps; /* FP64-contraction i k gather: warps per tile, 2, 4 or 8,
                       each with 64 / (8 warps) blocks of 8 atoms per round
                       (default 4) */
  int stencil;      /* mixed form's spread and gathers: 1 the FP64 tensor cores
                       on its FP32 weights and grids (default), 2 FP32 CUDA cores */
} ewg_kernel_shape;

/* Kernel-shape autotuner.  Evaluates the caller's configuration (the
 * parameters the reference chain gives for tol, or the overrides) with the
 * context's form and force scheme, and searches the kernel shapes one field
 * at a time (box_div, stencil, gather_warps, fft_lines, fft_sched), keeping a change
 * only when the median of seven timed evaluations (graph replays) improves by
 * more than 1%.  The result is cached in the context per bucket -- precision
 * form, force grids (i k, window derivatives or potential only), atom count
 * by octave (2^k <= n < 2^(k+1)), fine grid and window half-width -- and every
 * later evaluation that falls in the bucket runs it.  out (may be NULL) gets the
 * shape; ms (optional, 2 doubles) the median milliseconds per evaluation with
 * the default shapes and with the chosen ones.  A bucket already tuned returns
 * its cached shape with ms[0] = ms[1] = 0 and evaluates nothing.
 * No counterpart in the reference. */
int ewg_tune_kernels(ewg_context* ctx, int n, const double* positions, const double* charges,
                     const double* lat_rows, double tol, const ewg_overrides* ov,
                     int want_force, ewg_kernel_shape* out, double* ms);
/* Pin the kernel shapes of every later evaluation of the context (zero fields:
 * defaults); NULL returns to the tuned buckets and the defaults. */
int ewg_set_kernel_shape(ewg_context* ctx, const ewg_kernel_shape* shape);

/* ewald_parameters (fft/ewald_fft_3d.f90:142-191); host only. */
int ewg_parameters(int n, const double* charges, const double* lat_rows, double tol,
                   const ewg_overrides* ov, ewg_params* out);

/* ewald_grid_memory (fft/ewald_fft_3d.f90:197-244) in the reference's own
 * accounting (complex fine grid plus two mode arrays, GiB); host only. */
int ewg_grid_memory(int n, const double* charges, const double* lat_rows, double tol,
                    const ewg_overrides* ov, double* gigabytes);

/* Device bytes this library would hold for such an evaluation (all buffers of
 * the chosen precision), so that a caller can gate a size sweep. */
int ewg_device_memory(int n, const double* charges, const double* lat_rows, double tol,
                      const ewg_overrides* ov, int precision, int with_force, double* bytes);

/* Same as ewg_potential_force with every array already in device memory:
 * coords(3,N), charges(N), pot(N), force(3,N) all device pointers; lat_rows on
 * the host.  The charge sums the parameter chain needs are reduced on the GPU
 * and read back (24 bytes).  When ov fixes alpha and k_cut (as ewg_tune's
 * result does) and the background convention is off, the parameters do not
 * depend on the charges: the evaluation is queued without waiting for the
 * sums, and the neutrality check (EWG_ERR_NOT_NEUTRAL) is made after it, once
 * the call has synchronised. */
int ewg_potential_force_device(ewg_context* ctx, int n, const double* coords_device,
                               const double* charges_device, const double* lat_rows, double tol,
                               double* pot_device, double* force_device, const ewg_overrides* ov);

/* ---- library surface: direct/ewald_direct_3d.f90 ------------------------ */

/* ewald_potential_force of the direct O(N^2) engine (direct/ewald_direct_3d.f90:37-182):
 * balanced splitting (common/ewald_alpha_search.f90:83-181), explicit image sum
 * and a direct structure-factor sum over the k sphere.  The optional
 * arguments are NULL when absent. */
int ewg_direct_potential_force(ewg_context* ctx, int n, const double* positions,
                               const double* charges, const double* lat_rows, double tol,
                               double* pot, double* force, const double* alpha_in,
                               const double* r_cut_in, const double* k_cut_in);

/* The direct engine without any allocation.  No counterpart in the reference:
 * it exists for host codes that cannot allocate device memory once a run is
 * under way (for instance a program that gives all device memory to its own
 * pool allocator at start-up, or one that must not risk an allocation failing
 * or stalling inside an MD or SCC loop).  Same results as
 * ewg_direct_potential_force, but every array is a device pointer owned by the
 * caller: coords(3,N), charges(N), pot(N), force(3,N) (force may be NULL);
 * lat_rows and the optional arguments are host values.  All working memory
 * comes from one fixed 16 MiB array in device memory that every GPU loading
 * the library holds until the process exits; configurations that do not fit
 * (atoms, cell-list boxes and Fourier modes together) return
 * EWG_ERR_SCRATCH_LIMIT before any kernel runs.  It calls no cudaMalloc,
 * cudaFree or other allocating routine.  All calls share that array, so calls
 * that overlap on the GPU race; run them one at a time.  The first call on a
 * device looks up the array's device address for that device; make that first
 * call before any stream capture begins.  Under CUDA's lazy module loading (the
 * default since CUDA 12.2) that first call is also what reserves the 16 MiB on
 * the device, so a program that gives all device memory to its own pool must
 * make one small call on each device before its pool takes the memory (else
 * the first call can return EWG_ERR_OUT_OF_MEMORY).  stream is a cudaStream_t
 * (NULL: the default stream); the call returns after the work has finished. */
int ewg_direct_potential_force_static(int n, const double* coords_device,
                                      const double* charges_device, const double* lat_rows,
                                      double tol, double* pot_device, double* force_device,
                                      const double* alpha_in, const double* r_cut_in,
                                      const double* k_cut_in, void* stream);

/* ---- TCoulomb surface: src/dftbp/dftb/coulomb.F90 ----------------------- */

/* TCoulomb%updateLatVecs (coulomb.F90:575-620): lattice vectors as columns. */
int ewg_set_lattice(ewg_context* ctx, const double* lat_cols);
/* TCoulomb%updateCoords (coulomb.F90:509-572): coords(3,N) of the central cell.
 * Geometry-only device state (fractional coordinates, cell list, stencil
 * weights) is rebuilt lazily at the next evaluation and then kept resident. */
int ewg_set_coords(ewg_context* ctx, int n, const double* coords);
/* TCoulomb%updateCharges (coulomb.F90:760-781): deltaQAtom(N). */
int ewg_set_charges(ewg_context* ctx, const double* dq);
/* fftEwaldShift (coulomb.F90:336-357) inside TCoulomb%updateShifts (:786-880):
 * shift(N) = per-atom potential.  tol <= 0 or >= 1 selects 1e-9 as the
 * adapter does (:348-349). */
int ewg_shift(ewg_context* ctx, double tol, double* shift);
/* fftEwaldAddGradients (coulomb.F90:361-385): shift(N) and the physical force
 * F(3,N); the adapter subtracts F from DFTB+'s gradient array. */
int ewg_shift_force(ewg_context* ctx, double tol, double* shift, double* force);
/* k charge updates on the resident geometry in one submission: for each j,
 * the result of ewg_set_charges(charges + j N) then ewg_shift(tol, shifts + j N)
 * (updateCharges, coulomb.F90:760-781, then fftEwaldShift, :336-357), bitwise,
 * each update with its own parameters from its own charges.  charges and
 * shifts are (N, k) column-major (update-major); one upload, one download and
 * no host wait between the updates.  Afterwards the context's charges are the
 * last update's.  Returns the first failing check (every update is checked
 * before any work is queued; nothing is written then) or EWG_ERR_COINCIDENT
 * (shifts written all the same).  No counterpart in the reference, whose SCC
 * loop calls the shift once per iteration. */
int ewg_shift_batch(ewg_context* ctx, double tol, int k, const double* charges, double* shifts);
/* ---- potentials and gradients at arbitrary points ---------------------- */
/* TCoulomb%getPotential / getPotentialGradient / addExternalPotGrad
 * (dftb/coulomb.F90:3122-3248), periodic branch: the stock Ewald sum of
 * sumInvRPeriodicAsymm (:1340-1418) and addInvRPrimePeriodicAsymm (:1934-2092)
 * between two point sets, with updateLatVecs's setup (:575-620) for the given
 * lattice (one vector per column), tolerance and alpha (<= 0 selects
 * getOptimalAlphaEwald).  Coordinates are (3, n) column-major (atom-major),
 * gradients likewise.  blur_widths (Gaussian width of each source or external
 * charge) and eps_soften (a pointer to the softening length) may be NULL. */
int ewg_potential_at(ewg_context* ctx, int n_targets, const double* target_coords, int n_sources,
                     const double* source_coords, const double* source_charges,
                     const double* blur_widths, const double* eps_soften, const double* lat_cols,
                     double tol_ewald, double alpha, double* potential);
int ewg_potential_gradient_at(ewg_context* ctx, int n_targets, const double* target_coords,
                              int n_sources, const double* source_coords,
                              const double* source_charges, const double* blur_widths,
                              const double* lat_cols, double tol_ewald, double alpha,
                              double* gradient);
/* Adds to atom_grads (and, unless ham_deriv, to ext_grads) like the reference
 * (intent inout); ham_deriv != 0 gives the Hamiltonian derivative (no atom
 * charges, ext_grads untouched). */
int ewg_external_pot_grad(ewg_context* ctx, int n_atoms, const double* atom_coords, int n_ext,
                          const double* ext_coords, const double* atom_charges,
                          const double* ext_charges, int ham_deriv, const double* ext_blur_widths,
                          const double* lat_cols, double tol_ewald, double alpha,
                          double* atom_grads, double* ext_grads);

/* XLBOMD gradients (addGradients with dQOutAtom, coulomb.F90:697-699): adds to
 * gradients(3, N) the gradient of the shadow energy
 * sum_{i<j} (qo_i qi_j + qi_i qo_j - qi_i qi_j) phi(r_ij) with qi the charges set
 * by ewg_set_charges and qo = dq_out.  The reference sums it with the stock
 * Ewald engine (addInvRPrimeXlbomdPeriodic, :1823-1894); here it is the fast
 * path's energy gradient of E(qi + qo) - E(qo) - 2 E(qi), three evaluations on
 * the resident geometry with one parameter set (tol as in ewg_shift_force).
 * Both charge sets must be neutral (EWG_ERR_NOT_NEUTRAL otherwise). */
int ewg_xlbomd_gradients(ewg_context* ctx, double tol, const double* dq_out, double* gradients);

/* The NFFT-based stress of ewg_potential_force_stress on the state set by
 * ewg_set_lattice / ewg_set_coords / ewg_set_charges (the fast path's own alpha
 * and cutoffs at tolerance tol, <= 0 or >= 1 meaning 1e-9 as in fftEwaldShift):
 * sigma = (2/V) dE/d(strain), the invRStress convention, so addStress can do
 * stress -= 0.5 sigma with it instead of the stock engine.  Reuses the resident
 * geometry like ewg_shift.  No counterpart in the reference (its next step for
 * the fast path, fft3d_readme.md:30). */
int ewg_stress_fast(ewg_context* ctx, double tol, double* sigma);

/* invRStress (coulomb.F90:2777-2863) with the stock setup of updateLatVecs
 * (getOptimalAlphaEwald when alpha <= 0, getMaxREwald, getMaxGEwald,
 * getLatticePoints): sigma(3,3) column-major; TCoulomb%addStress then does
 * stress -= 0.5*sigma (coulomb.F90:755). */
int ewg_stress(ewg_context* ctx, double tol_ewald, double alpha, double* sigma);
/* The splitting parameter, real cutoff, reciprocal cutoff and number of
 * half-space reciprocal vectors the last ewg_stress call used. */
int ewg_last_stress_setup(const ewg_context* ctx, double* alpha, double* max_r, double* max_g,
                          int* n_g);

/* ---- batched form ------------------------------------------------------- */

/* ewald_potential_force on many independent cells in one submission.
 * Cell c holds atoms [offsets[c], offsets[c+1]); coords(3, total) atom-major,
 * lat_rows 9 doubles per cell (Fortran rows layout); pot(total), force(3,total).
 * Each cell gets its own parameters from the reference chain.  Status of
 * cell c goes to cell_status[c] when cell_status is not NULL; the return value
 * is the first non-zero cell status.  By default every stage of every cell
 * runs in one segmented launch (the cells' parameters, FFT plans and buffers
 * in a device table), and a repeated batch is recorded as one CUDA graph and
 * replayed; cells whose real FFT grids average more than 64 MiB run one after
 * another instead (one such cell fills the GPU on its own).  With
 * ewg_set_batch_lanes(ctx, 1..16) the cells run on that many concurrent lanes.
 * Results are bitwise the same either way. */
int ewg_batch_potential_force(ewg_context* ctx, int n_cells, const int* offsets,
                              const double* coords, const double* charges, const double* lat_rows,
                              double tol, double* pot, double* force, int* cell_status);

/* The same with overrides applied to every cell (e.g. the result of ewg_tune
 * for a batch of like cells).  ov may be NULL.  No counterpart in the
 * reference. */
int ewg_batch_potential_force_ov(ewg_context* ctx, int n_cells, const int* offsets,
                                 const double* coords, const double* charges,
                                 const double* lat_rows, double tol, double* pot, double* force,
                                 int* cell_status, const ewg_overrides* ov);

/* Batch lanes (0..16, default 0).  0: segmented launches, one per stage for
 * all cells of a batched call (cells that fail their checks send the whole
 * call to the lane path, and cells whose real grids average more than 64 MiB
 * run one after another on the context).  1..16: independent cells run concurrently on this
 * many lanes, each a sub-context of the same device, form and settings with
 * its own device buffers and streams (so each lane holds the buffers of the
 * largest cell it has run); one lane runs the cells back to back on the
 * context itself.  No counterpart in the reference. */
int ewg_set_batch_lanes(ewg_context* ctx, int lanes);

#ifdef __cplusplus
}
#endif
#endif
