!> Fortran binding of the B200 Ewald operator's C ABI (include/ewald_b200.h).
!>
!> This module is what DFTB+ compiles next to src/dftbp/dftb/coulomb.F90 to
!> reach the GPU engine: bind(C) interfaces in the style of the reference's own
!> C interop (src/dftbp/common/envcheck.F90:24-38), plus thin wrappers that keep
!> the reference library's argument order and stop with the library's message
!> on a non-zero status, as the reference's `error stop` does.
!>
!> Arrays are passed in DFTB+'s native layouts: coords(3,N), latVecs(3,3) with
!> one lattice vector per column, force(3,N).  No transposes are needed.
module ewald_b200
  use, intrinsic :: iso_c_binding, only : c_int, c_double, c_ptr, c_null_ptr, c_char, &
      & c_associated, c_f_pointer, c_long_long, c_loc
  implicit none
  private

  public :: TEwaldGpu, ewaldGpuInit, ewaldGpuFinal
  public :: ewaldGpuSetLattice, ewaldGpuSetCoords, ewaldGpuSetCharges
  public :: ewaldGpuShift, ewaldGpuShiftForce, ewaldGpuStress, ewaldGpuStressFast
  public :: ewaldGpuShiftBatch
  public :: ewaldGpuPotentialForce, ewaldGpuPotentialAt, ewaldGpuPotentialGradientAt
  public :: ewaldGpuSetForceScheme, ewaldGpuSetBackground, ewaldGpuXlbomdGradients
  public :: ewaldGpuExternalPotGrad, ewaldGpuPotentialForceStress, ewaldGpuBatchPotentialForce
  public :: ewaldGpuSetPointEngine, ewaldGpuTuneKernels, ewaldGpuSetKernelShape, TEwgKernelShape
  public :: ewaldGpuParameters, ewaldGpuGridMemory, ewaldGpuLastParams, ewaldGpuTune
  public :: ewaldGpuDirectPotentialForce, TEwgParams, TEwgOverrides
  public :: EWG_PRECISION_FP64, EWG_PRECISION_MIXED, EWG_FORCE_IK, EWG_FORCE_AD
  public :: EWG_POINTS_AUTO, EWG_POINTS_STOCK, EWG_POINTS_MESH

  integer(c_int), parameter :: EWG_PRECISION_FP64 = 0
  integer(c_int), parameter :: EWG_PRECISION_MIXED = 1
  integer(c_int), parameter :: EWG_FORCE_IK = 0
  integer(c_int), parameter :: EWG_FORCE_AD = 1
  integer(c_int), parameter :: EWG_POINTS_AUTO = 0
  integer(c_int), parameter :: EWG_POINTS_STOCK = 1
  integer(c_int), parameter :: EWG_POINTS_MESH = 2

  !> Handle of one device context.
  type :: TEwaldGpu
    type(c_ptr) :: ctx = c_null_ptr
  end type TEwaldGpu

  !> ewg_overrides of the C header (unused members carry has_* = 0).
  type, bind(C) :: TEwgOverrides
    integer(c_int) :: has_alpha = 0, has_r_cut = 0, has_k_cut = 0, has_n_modes = 0, &
        & has_window_cutoff = 0
    real(c_double) :: alpha = 0.0_c_double, r_cut = 0.0_c_double, k_cut = 0.0_c_double
    integer(c_int) :: n_modes = 0, window_cutoff = 0
  end type TEwgOverrides

  !> ewg_params of the C header: TEwaldParameters3d
  !> (fft/ewald_fft_3d_parameters.f90:24-42).
  type, bind(C) :: TEwgParams
    real(c_double) :: alpha = 0.0_c_double, r_cut = 0.0_c_double, k_cut = 0.0_c_double
    integer(c_int) :: window_cutoff = 0
    integer(c_int) :: n_modes(3) = 0
  end type TEwgParams

  !> ewg_kernel_shape of the C header (0 = the library's default).
  type, bind(C) :: TEwgKernelShape
    integer(c_int) :: box_div = 0, fft_lines = 0, fft_sched = 0, gather_warps = 0, stencil = 0
  end type TEwgKernelShape

  interface
    function ewg_create(ctx, device, precision) bind(C, name="ewg_create") result(rc)
      import :: c_ptr, c_int
      type(c_ptr), intent(out) :: ctx
      integer(c_int), value :: device, precision
      integer(c_int) :: rc
    end function ewg_create

    function ewg_destroy(ctx) bind(C, name="ewg_destroy") result(rc)
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int) :: rc
    end function ewg_destroy

    function ewg_status_string(status) bind(C, name="ewg_status_string") result(msg)
      import :: c_int, c_ptr
      integer(c_int), value :: status
      type(c_ptr) :: msg
    end function ewg_status_string

    function ewg_set_lattice(ctx, latCols) bind(C, name="ewg_set_lattice") result(rc)
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: latCols(3, 3)
      integer(c_int) :: rc
    end function ewg_set_lattice

    function ewg_set_coords(ctx, n, coords) bind(C, name="ewg_set_coords") result(rc)
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: n
      real(c_double), intent(in) :: coords(3, *)
      integer(c_int) :: rc
    end function ewg_set_coords

    function ewg_set_charges(ctx, dq) bind(C, name="ewg_set_charges") result(rc)
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: dq(*)
      integer(c_int) :: rc
    end function ewg_set_charges

    function ewg_shift(ctx, tol, shift) bind(C, name="ewg_shift") result(rc)
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: tol
      real(c_double), intent(out) :: shift(*)
      integer(c_int) :: rc
    end function ewg_shift

    function ewg_shift_force(ctx, tol, shift, force) bind(C, name="ewg_shift_force") result(rc)
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: tol
      real(c_double), intent(out) :: shift(*)
      real(c_double), intent(out) :: force(3, *)
      integer(c_int) :: rc
    end function ewg_shift_force

    function ewg_shift_batch(ctx, tol, k, charges, shifts) bind(C, name="ewg_shift_batch") &
        & result(rc)
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: tol
      integer(c_int), value :: k
      real(c_double), intent(in) :: charges(*)
      real(c_double), intent(out) :: shifts(*)
      integer(c_int) :: rc
    end function ewg_shift_batch

    function ewg_stress(ctx, tolEwald, alpha, sigma) bind(C, name="ewg_stress") result(rc)
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: tolEwald, alpha
      real(c_double), intent(out) :: sigma(3, 3)
      integer(c_int) :: rc
    end function ewg_stress

    function ewg_set_force_scheme(ctx, scheme) bind(C, name="ewg_set_force_scheme") result(rc)
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int), value :: scheme
      integer(c_int) :: rc
    end function ewg_set_force_scheme

    function ewg_tune_kernels(ctx, n, positions, charges, latRows, tol, ov, wantForce, shape, ms) &
        & bind(C, name="ewg_tune_kernels") result(rc)
      import :: c_ptr, c_int, c_double, TEwgOverrides, TEwgKernelShape
      type(c_ptr), value :: ctx
      integer(c_int), value :: n, wantForce
      real(c_double), intent(in) :: positions(n, 3), charges(n), latRows(3, 3)
      real(c_double), value :: tol
      type(TEwgOverrides), intent(in) :: ov
      type(TEwgKernelShape), intent(out) :: shape
      real(c_double), intent(out) :: ms(2)
      integer(c_int) :: rc
    end function ewg_tune_kernels

    function ewg_set_kernel_shape(ctx, shape) bind(C, name="ewg_set_kernel_shape") result(rc)
      import :: c_ptr, c_int, TEwgKernelShape
      type(c_ptr), value :: ctx
      type(TEwgKernelShape), intent(in) :: shape
      integer(c_int) :: rc
    end function ewg_set_kernel_shape

    function ewg_parameters(n, charges, latRows, tol, ov, params) &
        & bind(C, name="ewg_parameters") result(rc)
      import :: c_int, c_double, TEwgOverrides, TEwgParams
      integer(c_int), value :: n
      real(c_double), intent(in) :: charges(n), latRows(3, 3)
      real(c_double), value :: tol
      type(TEwgOverrides), intent(in) :: ov
      type(TEwgParams), intent(out) :: params
      integer(c_int) :: rc
    end function ewg_parameters

    function ewg_grid_memory(n, charges, latRows, tol, ov, gigabytes) &
        & bind(C, name="ewg_grid_memory") result(rc)
      import :: c_int, c_double, TEwgOverrides
      integer(c_int), value :: n
      real(c_double), intent(in) :: charges(n), latRows(3, 3)
      real(c_double), value :: tol
      type(TEwgOverrides), intent(in) :: ov
      real(c_double), intent(out) :: gigabytes
      integer(c_int) :: rc
    end function ewg_grid_memory

    function ewg_last_params(ctx, params) bind(C, name="ewg_last_params") result(rc)
      import :: c_ptr, c_int, TEwgParams
      type(c_ptr), value :: ctx
      type(TEwgParams), intent(out) :: params
      integer(c_int) :: rc
    end function ewg_last_params

    function ewg_direct_potential_force(ctx, n, positions, charges, latRows, tol, pot, force, &
        & alphaIn, rCutIn, kCutIn) bind(C, name="ewg_direct_potential_force") result(rc)
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: n
      real(c_double), intent(in) :: positions(n, 3), charges(n), latRows(3, 3)
      real(c_double), value :: tol
      real(c_double), intent(out) :: pot(n), force(3, n)
      type(c_ptr), value :: alphaIn, rCutIn, kCutIn
      integer(c_int) :: rc
    end function ewg_direct_potential_force

    function ewg_tune(ctx, n, positions, charges, latRows, target, ov, scheme, report) &
        & bind(C, name="ewg_tune") result(rc)
      import :: c_ptr, c_int, c_double, TEwgOverrides
      type(c_ptr), value :: ctx
      integer(c_int), value :: n
      real(c_double), intent(in) :: positions(n, 3), charges(n), latRows(3, 3)
      real(c_double), value :: target
      type(TEwgOverrides), intent(out) :: ov
      integer(c_int), intent(out) :: scheme
      real(c_double), intent(out) :: report(4)
      integer(c_int) :: rc
    end function ewg_tune

    function ewg_set_point_engine(ctx, engine) bind(C, name="ewg_set_point_engine") result(rc)
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int), value :: engine
      integer(c_int) :: rc
    end function ewg_set_point_engine

    function ewg_stress_fast(ctx, tol, sigma) bind(C, name="ewg_stress_fast") result(rc)
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: tol
      real(c_double), intent(out) :: sigma(3, 3)
      integer(c_int) :: rc
    end function ewg_stress_fast

    function ewg_set_background(ctx, on) bind(C, name="ewg_set_background") result(rc)
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int), value :: on
      integer(c_int) :: rc
    end function ewg_set_background

    function ewg_xlbomd_gradients(ctx, tol, dqOut, gradients) &
        & bind(C, name="ewg_xlbomd_gradients") result(rc)
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: tol
      real(c_double), intent(in) :: dqOut(*)
      real(c_double), intent(inout) :: gradients(3, *)
      integer(c_int) :: rc
    end function ewg_xlbomd_gradients

    function ewg_external_pot_grad(ctx, na, acoords, ne, ecoords, acharges, echarges, hamDeriv,&
        & blur, latVecs, tolEwald, alpha, atomGrads, extGrads)&
        & bind(C, name="ewg_external_pot_grad") result(rc)
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: na, ne, hamDeriv
      real(c_double), intent(in) :: acoords(3, na), ecoords(3, ne), latVecs(3, 3)
      type(c_ptr), value :: acharges, blur, extGrads
      real(c_double), intent(in) :: echarges(ne)
      real(c_double), value :: tolEwald, alpha
      real(c_double), intent(inout) :: atomGrads(3, na)
      integer(c_int) :: rc
    end function ewg_external_pot_grad

    function ewg_potential_force_stress(ctx, n, positions, charges, latRows, tol, pot, force,&
        & sigma, ov) bind(C, name="ewg_potential_force_stress") result(rc)
      import :: c_ptr, c_int, c_double, TEwgOverrides
      type(c_ptr), value :: ctx
      integer(c_int), value :: n
      real(c_double), intent(in) :: positions(n, 3), charges(n), latRows(3, 3)
      real(c_double), value :: tol
      real(c_double), intent(out) :: pot(n), force(3, n), sigma(3, 3)
      type(TEwgOverrides), intent(in) :: ov
      integer(c_int) :: rc
    end function ewg_potential_force_stress

    function ewg_batch_potential_force_ov(ctx, nCells, offsets, coords, charges, latRows, tol,&
        & pot, force, cellStatus, ov) bind(C, name="ewg_batch_potential_force_ov") result(rc)
      import :: c_ptr, c_int, c_double, TEwgOverrides
      type(c_ptr), value :: ctx
      integer(c_int), value :: nCells
      integer(c_int), intent(in) :: offsets(nCells + 1)
      real(c_double), intent(in) :: coords(3, *), charges(*), latRows(9, nCells)
      real(c_double), value :: tol
      real(c_double), intent(out) :: pot(*), force(3, *)
      integer(c_int), intent(out) :: cellStatus(nCells)
      type(TEwgOverrides), intent(in) :: ov
      integer(c_int) :: rc
    end function ewg_batch_potential_force_ov

    function ewg_potential_at(ctx, nt, tcoords, ns, scoords, scharges, blur, epsSoften, latVecs,&
        & tolEwald, alpha, pot) bind(C, name="ewg_potential_at") result(rc)
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: nt, ns
      real(c_double), intent(in) :: tcoords(3, nt), scoords(3, ns), scharges(ns), latVecs(3, 3)
      type(c_ptr), value :: blur, epsSoften
      real(c_double), value :: tolEwald, alpha
      real(c_double), intent(out) :: pot(nt)
      integer(c_int) :: rc
    end function ewg_potential_at

    function ewg_potential_gradient_at(ctx, nt, tcoords, ns, scoords, scharges, blur, latVecs,&
        & tolEwald, alpha, grad) bind(C, name="ewg_potential_gradient_at") result(rc)
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: nt, ns
      real(c_double), intent(in) :: tcoords(3, nt), scoords(3, ns), scharges(ns), latVecs(3, 3)
      type(c_ptr), value :: blur
      real(c_double), value :: tolEwald, alpha
      real(c_double), intent(out) :: grad(3, nt)
      integer(c_int) :: rc
    end function ewg_potential_gradient_at

    function ewg_potential_force(ctx, n, positions, charges, latRows, tol, pot, force, ov) &
        & bind(C, name="ewg_potential_force") result(rc)
      import :: c_ptr, c_int, c_double, TEwgOverrides
      type(c_ptr), value :: ctx
      integer(c_int), value :: n
      real(c_double), intent(in) :: positions(n, 3), charges(n), latRows(3, 3)
      real(c_double), value :: tol
      real(c_double), intent(out) :: pot(n)
      real(c_double), intent(out) :: force(3, n)
      type(TEwgOverrides), intent(in) :: ov
      integer(c_int) :: rc
    end function ewg_potential_force
  end interface

contains

  !> Stop with the library's message, as the reference does on invalid input.
  subroutine check(rc)
    integer(c_int), intent(in) :: rc
    character(kind=c_char), pointer :: msg(:)
    character(len=128) :: text
    integer :: i
    if (rc == 0) return
    call c_f_pointer(ewg_status_string(rc), msg, [128])
    text = ""
    do i = 1, 128
      if (msg(i) == achar(0)) exit
      text(i:i) = msg(i)
    end do
    error stop trim(text)
  end subroutine check

  subroutine ewaldGpuInit(this, device, precision)
    type(TEwaldGpu), intent(out) :: this
    integer, intent(in), optional :: device, precision
    integer(c_int) :: dev, prec
    dev = 0
    prec = EWG_PRECISION_FP64
    if (present(device)) dev = device
    if (present(precision)) prec = precision
    call check(ewg_create(this%ctx, dev, prec))
  end subroutine ewaldGpuInit

  subroutine ewaldGpuFinal(this)
    type(TEwaldGpu), intent(inout) :: this
    if (c_associated(this%ctx)) call check(ewg_destroy(this%ctx))
    this%ctx = c_null_ptr
  end subroutine ewaldGpuFinal

  !> TCoulomb%updateLatVecs (coulomb.F90:575): latVecs(:, i) = a_i.
  subroutine ewaldGpuSetLattice(this, latVecs)
    type(TEwaldGpu), intent(in) :: this
    real(c_double), intent(in) :: latVecs(3, 3)
    call check(ewg_set_lattice(this%ctx, latVecs))
  end subroutine ewaldGpuSetLattice

  !> TCoulomb%updateCoords (coulomb.F90:509): coords(3, N) of the central cell.
  subroutine ewaldGpuSetCoords(this, coords)
    type(TEwaldGpu), intent(in) :: this
    real(c_double), intent(in) :: coords(:, :)
    call check(ewg_set_coords(this%ctx, int(size(coords, 2), c_int), coords))
  end subroutine ewaldGpuSetCoords

  !> TCoulomb%updateCharges (coulomb.F90:760).
  subroutine ewaldGpuSetCharges(this, deltaQAtom)
    type(TEwaldGpu), intent(in) :: this
    real(c_double), intent(in) :: deltaQAtom(:)
    call check(ewg_set_charges(this%ctx, deltaQAtom))
  end subroutine ewaldGpuSetCharges

  !> Replaces the call in fftEwaldShift (coulomb.F90:355).
  subroutine ewaldGpuShift(this, tol, shift)
    type(TEwaldGpu), intent(in) :: this
    real(c_double), intent(in) :: tol
    real(c_double), intent(out) :: shift(:)
    call check(ewg_shift(this%ctx, tol, shift))
  end subroutine ewaldGpuShift

  !> Replaces the call in fftEwaldAddGradients (coulomb.F90:380); force = -dU/dR.
  subroutine ewaldGpuShiftForce(this, tol, shift, force)
    type(TEwaldGpu), intent(in) :: this
    real(c_double), intent(in) :: tol
    real(c_double), intent(out) :: shift(:), force(:, :)
    call check(ewg_shift_force(this%ctx, tol, shift, force))
  end subroutine ewaldGpuShiftForce

  !> k charge updates on the resident geometry in one submission: column j of
  !> shifts is what ewaldGpuSetCharges(charges(:, j)) and ewaldGpuShift would give.
  subroutine ewaldGpuShiftBatch(this, tol, charges, shifts)
    type(TEwaldGpu), intent(inout) :: this
    real(c_double), intent(in) :: tol
    real(c_double), intent(in) :: charges(:, :)
    real(c_double), intent(out) :: shifts(:, :)
    call check(ewg_shift_batch(this%ctx, tol, int(size(charges, 2), c_int), charges, shifts))
  end subroutine ewaldGpuShiftBatch

  !> Replaces invRStress in TCoulomb%addStress (coulomb.F90:752); the caller
  !> keeps stress = stress - 0.5 * sigma.
  subroutine ewaldGpuStress(this, tolEwald, alpha, sigma)
    type(TEwaldGpu), intent(in) :: this
    real(c_double), intent(in) :: tolEwald, alpha
    real(c_double), intent(out) :: sigma(3, 3)
    call check(ewg_stress(this%ctx, tolEwald, alpha, sigma))
  end subroutine ewaldGpuStress

  !> Force differentiation scheme: EWG_FORCE_IK, the reference's i k (default),
  !> or EWG_FORCE_AD, window derivatives (one inverse transform instead of four).
  subroutine ewaldGpuSetForceScheme(this, scheme)
    type(TEwaldGpu), intent(inout) :: this
    integer(c_int), intent(in) :: scheme
    call check(ewg_set_force_scheme(this%ctx, scheme))
  end subroutine ewaldGpuSetForceScheme

  !> Kernel-shape autotuner for the bucket of this configuration (precision
  !> form, force grids, atom octave, grid, window); called once, for example
  !> after the first updateCoords, so that the SCC loop's evaluations run the
  !> fastest shapes. ms (optional) gets the default and tuned milliseconds.
  subroutine ewaldGpuTuneKernels(this, positions, charges, latRows, tol, wantForce, shape, ms)
    type(TEwaldGpu), intent(inout) :: this
    real(c_double), intent(in) :: positions(:, :), charges(:), latRows(3, 3), tol
    logical, intent(in) :: wantForce
    type(TEwgKernelShape), intent(out) :: shape
    real(c_double), intent(out), optional :: ms(2)
    type(TEwgOverrides) :: ov
    real(c_double) :: msLoc(2)
    integer(c_int) :: wf
    wf = 0
    if (wantForce) wf = 1
    call check(ewg_tune_kernels(this%ctx, int(size(charges), c_int), positions, charges, latRows, &
        & tol, ov, wf, shape, msLoc))
    if (present(ms)) ms = msLoc
  end subroutine ewaldGpuTuneKernels

  !> Pin kernel shapes for every later evaluation (zero fields: defaults).
  subroutine ewaldGpuSetKernelShape(this, shape)
    type(TEwaldGpu), intent(inout) :: this
    type(TEwgKernelShape), intent(in) :: shape
    call check(ewg_set_kernel_shape(this%ctx, shape))
  end subroutine ewaldGpuSetKernelShape

  !> ewald_parameters (fft/ewald_fft_3d.f90:142-191): the parameter set the
  !> reference chain selects for these charges, cell and tolerance (host only).
  subroutine ewaldGpuParameters(charges, nParticle, latVecs, tol, params)
    real(c_double), intent(in) :: charges(:), latVecs(3, 3), tol
    integer, intent(in) :: nParticle
    type(TEwgParams), intent(out) :: params
    type(TEwgOverrides) :: ov
    call check(ewg_parameters(int(nParticle, c_int), charges, latVecs, tol, ov, params))
  end subroutine ewaldGpuParameters

  !> ewald_grid_memory (fft/ewald_fft_3d.f90:197-244): GiB in the reference's
  !> own accounting (host only).
  function ewaldGpuGridMemory(charges, nParticle, latVecs, tol) result(gib)
    real(c_double), intent(in) :: charges(:), latVecs(3, 3), tol
    integer, intent(in) :: nParticle
    real(c_double) :: gib
    type(TEwgOverrides) :: ov
    call check(ewg_grid_memory(int(nParticle, c_int), charges, latVecs, tol, ov, gib))
  end function ewaldGpuGridMemory

  !> Parameters of the context's last evaluation (alpha, cutoffs, window, modes).
  subroutine ewaldGpuLastParams(this, params)
    type(TEwaldGpu), intent(in) :: this
    type(TEwgParams), intent(out) :: params
    call check(ewg_last_params(this%ctx, params))
  end subroutine ewaldGpuLastParams

  !> The direct engine (direct/ewald_direct_3d.f90:37-182), which the adapter
  !> takes under DFTB_EWALD_DIRECT=1; alpha, rCut and kCut default to the
  !> engine's own balance when absent.
  subroutine ewaldGpuDirectPotentialForce(this, positions, charges, nParticle, latVecs, tol, pot, &
      & force, alpha, rCut, kCut)
    type(TEwaldGpu), intent(in) :: this
    real(c_double), intent(in) :: positions(:, :), charges(:), latVecs(3, 3), tol
    integer, intent(in) :: nParticle
    real(c_double), intent(out) :: pot(:), force(:, :)
    real(c_double), intent(in), optional, target :: alpha, rCut, kCut
    type(c_ptr) :: pAlpha, pRCut, pKCut
    pAlpha = c_null_ptr
    pRCut = c_null_ptr
    pKCut = c_null_ptr
    if (present(alpha)) pAlpha = c_loc(alpha)
    if (present(rCut)) pRCut = c_loc(rCut)
    if (present(kCut)) pKCut = c_loc(kCut)
    call check(ewg_direct_potential_force(this%ctx, int(nParticle, c_int), positions, charges, &
        & latVecs, tol, pot, force, pAlpha, pRCut, pKCut))
  end subroutine ewaldGpuDirectPotentialForce

  !> Parameter autotuner of the context's form: the overrides and force scheme
  !> of the fastest candidate within the RMS error bar set by target; report
  !> (optional) gets its force and potential RMS errors, milliseconds per
  !> evaluation and the number of candidates evaluated.
  subroutine ewaldGpuTune(this, positions, charges, latVecs, target, ov, scheme, report)
    type(TEwaldGpu), intent(inout) :: this
    real(c_double), intent(in) :: positions(:, :), charges(:), latVecs(3, 3), target
    type(TEwgOverrides), intent(out) :: ov
    integer(c_int), intent(out) :: scheme
    real(c_double), intent(out), optional :: report(4)
    real(c_double) :: rep(4)
    call check(ewg_tune(this%ctx, int(size(charges), c_int), positions, charges, latVecs, target, &
        & ov, scheme, rep))
    if (present(report)) report = rep
  end subroutine ewaldGpuTune

  !> Engine of ewaldGpuPotentialAt, ewaldGpuPotentialGradientAt and
  !> ewaldGpuExternalPotGrad: EWG_POINTS_STOCK (the stock pair sum of
  !> coulomb.F90:2311-2343), EWG_POINTS_MESH (NFFT plus a cell-list real-space
  !> sum, linear in the number of points) or EWG_POINTS_AUTO (mesh from 2**20
  !> target-source pairs on). Softened calls always take the stock sum.
  subroutine ewaldGpuSetPointEngine(this, engine)
    type(TEwaldGpu), intent(inout) :: this
    integer(c_int), intent(in) :: engine
    call check(ewg_set_point_engine(this%ctx, engine))
  end subroutine ewaldGpuSetPointEngine

  !> NFFT-based stress of the fast engine on the resident state; same convention as
  !> ewaldGpuStress (the caller does stress = stress - 0.5 * sigma).
  subroutine ewaldGpuStressFast(this, tol, sigma)
    type(TEwaldGpu), intent(in) :: this
    real(c_double), intent(in) :: tol
    real(c_double), intent(out) :: sigma(3, 3)
    call check(ewg_stress_fast(this%ctx, tol, sigma))
  end subroutine ewaldGpuStressFast

  !> TCoulomb%getPotential (coulomb.F90:3122-3153), with the optional Gaussian
  !> blur of each charge and the softening length.
  subroutine ewaldGpuPotentialAt(this, coords, chargeCoords, charges, latVecs, tolEwald, alpha,&
      & potential, blurWidths, epsSoften)
    type(TEwaldGpu), intent(in) :: this
    real(c_double), intent(in) :: coords(:, :), chargeCoords(:, :), charges(:), latVecs(3, 3)
    real(c_double), intent(in) :: tolEwald, alpha
    real(c_double), intent(out) :: potential(:)
    real(c_double), intent(in), optional, target, contiguous :: blurWidths(:)
    real(c_double), intent(in), optional, target :: epsSoften
    type(c_ptr) :: pBlur, pEps
    pBlur = c_null_ptr
    pEps = c_null_ptr
    if (present(blurWidths)) pBlur = c_loc(blurWidths)
    if (present(epsSoften)) pEps = c_loc(epsSoften)
    call check(ewg_potential_at(this%ctx, int(size(coords, 2), c_int), coords,&
        & int(size(chargeCoords, 2), c_int), chargeCoords, charges, pBlur, pEps,&
        & latVecs, tolEwald, alpha, potential))
  end subroutine ewaldGpuPotentialAt

  !> TCoulomb%getPotentialGradient (coulomb.F90:3157-3194), with the optional blur.
  subroutine ewaldGpuPotentialGradientAt(this, coords, chargeCoords, charges, latVecs, tolEwald,&
      & alpha, gradient, blurWidths)
    type(TEwaldGpu), intent(in) :: this
    real(c_double), intent(in) :: coords(:, :), chargeCoords(:, :), charges(:), latVecs(3, 3)
    real(c_double), intent(in) :: tolEwald, alpha
    real(c_double), intent(out) :: gradient(:, :)
    real(c_double), intent(in), optional, target, contiguous :: blurWidths(:)
    type(c_ptr) :: pBlur
    pBlur = c_null_ptr
    if (present(blurWidths)) pBlur = c_loc(blurWidths)
    call check(ewg_potential_gradient_at(this%ctx, int(size(coords, 2), c_int), coords,&
        & int(size(chargeCoords, 2), c_int), chargeCoords, charges, pBlur, latVecs, tolEwald,&
        & alpha, gradient))
  end subroutine ewaldGpuPotentialGradientAt

  !> TCoulomb%addExternalPotGrad (coulomb.F90:3198-3248).  Adds to atomGrads and,
  !> unless tHamDeriv, to extGrads (intent inout, like the reference); with
  !> tHamDeriv the atom charges are not used (pass any array) and extGrads is
  !> left untouched.
  subroutine ewaldGpuExternalPotGrad(this, atomCoords, extCoords, atomCharges, extCharges,&
      & tHamDeriv, latVecs, tolEwald, alpha, atomGrads, extGrads, extBlurWidths)
    type(TEwaldGpu), intent(in) :: this
    real(c_double), intent(in) :: atomCoords(:, :), extCoords(:, :), extCharges(:), latVecs(3, 3)
    real(c_double), intent(in), target, contiguous :: atomCharges(:)
    logical, intent(in) :: tHamDeriv
    real(c_double), intent(in) :: tolEwald, alpha
    real(c_double), intent(inout) :: atomGrads(:, :)
    real(c_double), intent(inout), target, contiguous :: extGrads(:, :)
    real(c_double), intent(in), optional, target, contiguous :: extBlurWidths(:)
    type(c_ptr) :: pBlur, pAtomQ, pExtGrads
    integer(c_int) :: hamDeriv
    pBlur = c_null_ptr
    if (present(extBlurWidths)) pBlur = c_loc(extBlurWidths)
    hamDeriv = 0
    pAtomQ = c_loc(atomCharges)
    pExtGrads = c_loc(extGrads)
    if (tHamDeriv) then
      hamDeriv = 1
      pAtomQ = c_null_ptr
      pExtGrads = c_null_ptr
    end if
    call check(ewg_external_pot_grad(this%ctx, int(size(atomCoords, 2), c_int), atomCoords,&
        & int(size(extCoords, 2), c_int), extCoords, pAtomQ, extCharges, hamDeriv, pBlur,&
        & latVecs, tolEwald, alpha, atomGrads, pExtGrads))
  end subroutine ewaldGpuExternalPotGrad

  !> Charged cells on the fast path with the stock engine's neutralising
  !> background (on = .true.); see ewg_set_background in the C header.
  subroutine ewaldGpuSetBackground(this, on)
    type(TEwaldGpu), intent(in) :: this
    logical, intent(in) :: on
    integer(c_int) :: flag
    flag = 0
    if (on) flag = 1
    call check(ewg_set_background(this%ctx, flag))
  end subroutine ewaldGpuSetBackground

  !> addGradients with dQOutAtom (coulomb.F90:697-699): adds the XLBOMD shadow
  !> energy's gradient to gradients(3, N), for the charges set by
  !> ewaldGpuSetCharges and dQOutAtom.
  subroutine ewaldGpuXlbomdGradients(this, tol, dQOutAtom, gradients)
    type(TEwaldGpu), intent(in) :: this
    real(c_double), intent(in) :: tol
    real(c_double), intent(in) :: dQOutAtom(:)
    real(c_double), intent(inout) :: gradients(:, :)
    call check(ewg_xlbomd_gradients(this%ctx, tol, dQOutAtom, gradients))
  end subroutine ewaldGpuXlbomdGradients

  !> ewald_potential_force plus the NFFT-based stress of the same evaluation
  !> (sigma in the invRStress convention: the caller does stress - 0.5 * sigma).
  subroutine ewaldGpuPotentialForceStress(this, positions, charges, nParticle, latVecs, tol, pot,&
      & force, sigma)
    type(TEwaldGpu), intent(in) :: this
    real(c_double), intent(in) :: positions(:, :), charges(:), latVecs(3, 3), tol
    integer, intent(in) :: nParticle
    real(c_double), intent(out) :: pot(:), force(:, :), sigma(3, 3)
    type(TEwgOverrides) :: ov
    call check(ewg_potential_force_stress(this%ctx, int(nParticle, c_int), positions, charges,&
        & latVecs, tol, pot, force, sigma, ov))
  end subroutine ewaldGpuPotentialForceStress

  !> ewald_potential_force on many independent cells in one submission: cell c
  !> holds atoms offsets(c)+1 .. offsets(c+1) (0-based CSR offsets, size nCells+1)
  !> of coords(3, :), latRows(:, c) its lattice in the rows layout of
  !> ewald_potential_force (column-major 3 x 3).  Stops on the first failing cell.
  subroutine ewaldGpuBatchPotentialForce(this, offsets, coords, charges, latRows, tol, pot, force)
    type(TEwaldGpu), intent(in) :: this
    integer(c_int), intent(in) :: offsets(:)
    real(c_double), intent(in) :: coords(:, :), charges(:), latRows(:, :), tol
    real(c_double), intent(out) :: pot(:), force(:, :)
    integer(c_int), allocatable :: cellStatus(:)
    type(TEwgOverrides) :: ov
    allocate(cellStatus(size(offsets) - 1))
    call check(ewg_batch_potential_force_ov(this%ctx, int(size(offsets) - 1, c_int), offsets,&
        & coords, charges, latRows, tol, pot, force, cellStatus, ov))
  end subroutine ewaldGpuBatchPotentialForce

  !> Same argument order as ewald_potential_force (fft/ewald_fft_3d.f90:36).
  subroutine ewaldGpuPotentialForce(this, positions, charges, nParticle, latVecs, tol, pot, force)
    type(TEwaldGpu), intent(in) :: this
    real(c_double), intent(in) :: positions(:, :), charges(:), latVecs(3, 3), tol
    integer, intent(in) :: nParticle
    real(c_double), intent(out) :: pot(:), force(:, :)
    type(TEwgOverrides) :: ov
    call check(ewg_potential_force(this%ctx, int(nParticle, c_int), positions, charges, latVecs, &
        & tol, pot, force, ov))
  end subroutine ewaldGpuPotentialForce

end module ewald_b200
