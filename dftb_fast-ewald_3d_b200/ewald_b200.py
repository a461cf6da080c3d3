"""Python host interface of the B200 Ewald operator (ctypes over libewald_b200.so).

It mirrors the reference's interfaces for the 3D-periodic Coulomb path:

* ``ewald_potential_force`` / ``ewald_parameters`` / ``ewald_grid_memory`` follow
  the fast library's public routines (src/dftbp/extlibs/fftewald/fft/ewald_fft_3d.f90:36-244):
  same argument names, ``positions(N,3)`` with one atom per row, lattice vectors
  as rows, tolerance default 1e-10, optional overrides ``alpha_in``,
  ``r_cut_in``, ``k_cut_in``, ``nModes_in``, ``windowCutoff_in``, and ``pot`` /
  ``force`` filled in place (``force`` is ``(3, N)`` as in Fortran).
* ``ewald_direct_potential_force`` follows the direct engine
  (direct/ewald_direct_3d.f90:37-182), default tolerance 1e-12.
* ``TCoulomb`` follows the type-bound procedures DFTB+'s SCC loop calls
  (src/dftbp/dftb/coulomb.F90:131-183): updateLatVecs, updateCoords,
  updateCharges, updateShifts, addShiftPerAtom, addEnergy, addGradients, addStress.

Where the reference stops with ``error stop``, this module raises
``EwaldError`` carrying the library's status code.  There is no CPU fallback:
if the CUDA library is missing or no GPU is present, calls fail loudly.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libewald_b200.so")

FP64 = 0
MIXED = 1
FORCE_IK = 0  # the reference's i k differentiation (the default)
FORCE_AD = 1  # analytic differentiation of the window
POINTS_AUTO = 0   # point potentials: mesh from 2^20 pairs on, stock below
POINTS_STOCK = 1  # the reference's stock pair sum, O(N_t N_s)
POINTS_MESH = 2   # NFFT + cell list, O(N_t + N_s)

STATUS = {
    0: "EWG_OK", 1: "EWG_ERR_NPARTICLE", 2: "EWG_ERR_ARG", 3: "EWG_ERR_NOT_NEUTRAL",
    4: "EWG_ERR_TOL", 5: "EWG_ERR_VOLUME", 6: "EWG_ERR_ALPHA", 7: "EWG_ERR_COINCIDENT",
    8: "EWG_ERR_CUTOFF", 9: "EWG_ERR_ALPHA_SEARCH", 10: "EWG_ERR_LATTICE_SEARCH",
    11: "EWG_ERR_OUT_OF_MEMORY", 12: "EWG_ERR_CUDA", 13: "EWG_ERR_DEVICE_TIMEOUT",
    14: "EWG_ERR_GRID_TOO_LARGE", 15: "EWG_ERR_NO_DEVICE", 16: "EWG_ERR_STATE",
    17: "EWG_ERR_SCRATCH_LIMIT",
}

# Every entry point of include/ewald_b200.h.
EXPORTED = [
    "ewg_create", "ewg_destroy", "ewg_status_string", "ewg_kernel_launches", "ewg_last_params",
    "ewg_potential_force", "ewg_parameters", "ewg_grid_memory", "ewg_device_memory",
    "ewg_potential_force_device", "ewg_direct_potential_force", "ewg_set_lattice",
    "ewg_set_coords", "ewg_set_charges", "ewg_shift", "ewg_shift_force", "ewg_shift_batch",
    "ewg_stress",
    "ewg_last_stress_setup", "ewg_batch_potential_force", "ewg_set_profiling", "ewg_stage_count",
    "ewg_stage_name", "ewg_stage_times", "ewg_reset_stage_times", "ewg_set_stream",
    "ewg_direct_potential_force_static", "ewg_fp64_mma_peak", "ewg_potential_force_stress",
    "ewg_stress_fast", "ewg_potential_at", "ewg_potential_gradient_at", "ewg_external_pot_grad",
    "ewg_xlbomd_gradients", "ewg_set_background", "ewg_set_force_scheme", "ewg_tune", "ewg_set_graphs", "ewg_set_batch_lanes",
    "ewg_batch_potential_force_ov", "ewg_set_point_engine", "ewg_tune_kernels",
    "ewg_set_kernel_shape",
]


class EwaldError(RuntimeError):
    """A non-zero status of the library; ``code`` is the EWG_* value."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{message} [{STATUS.get(code, code)}]")
        self.code = code


class Overrides(C.Structure):
    _fields_ = [
        ("has_alpha", C.c_int), ("has_r_cut", C.c_int), ("has_k_cut", C.c_int),
        ("has_n_modes", C.c_int), ("has_window_cutoff", C.c_int),
        ("alpha", C.c_double), ("r_cut", C.c_double), ("k_cut", C.c_double),
        ("n_modes", C.c_int), ("window_cutoff", C.c_int),
    ]


class KernelShape(C.Structure):
    """ewg_kernel_shape: kernel shapes of an evaluation (0 = the default)."""

    _fields_ = [("box_div", C.c_int), ("fft_lines", C.c_int), ("fft_sched", C.c_int),
                ("gather_warps", C.c_int), ("stencil", C.c_int)]

    def as_dict(self):
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


class Params(C.Structure):
    """TEwaldParameters3d (fft/ewald_fft_3d_parameters.f90:24-42)."""

    _fields_ = [("alpha", C.c_double), ("r_cut", C.c_double), ("k_cut", C.c_double),
                ("window_cutoff", C.c_int), ("n_modes", C.c_int * 3)]

    def as_dict(self):
        return {"alpha": self.alpha, "r_cut": self.r_cut, "k_cut": self.k_cut,
                "window_cutoff": self.window_cutoff, "n_modes": tuple(self.n_modes)}


_lib = None


def build(force: bool = False) -> str:
    import importlib.util

    spec = importlib.util.spec_from_file_location("_ewald_b200_build", os.path.join(HERE, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build(force=force)


def lib():
    """Load libewald_b200.so (raises OSError if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing: build it with build.py (no CPU fallback exists)")
    L = C.CDLL(LIB_PATH)
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    vp = C.c_void_p
    L.ewg_create.argtypes = [C.POINTER(vp), C.c_int, C.c_int]
    L.ewg_destroy.argtypes = [vp]
    L.ewg_status_string.argtypes = [C.c_int]
    L.ewg_status_string.restype = C.c_char_p
    L.ewg_kernel_launches.argtypes = [vp]
    L.ewg_kernel_launches.restype = C.c_longlong
    L.ewg_last_params.argtypes = [vp, C.POINTER(Params)]
    L.ewg_fp64_mma_peak.argtypes = [vp, dp]
    L.ewg_potential_force.argtypes = [vp, C.c_int, dp, dp, dp, C.c_double, dp, dp, C.POINTER(Overrides)]
    L.ewg_potential_force_stress.argtypes = [vp, C.c_int, dp, dp, dp, C.c_double, dp, dp, dp,
                                             C.POINTER(Overrides)]
    L.ewg_parameters.argtypes = [C.c_int, dp, dp, C.c_double, C.POINTER(Overrides), C.POINTER(Params)]
    L.ewg_tune.argtypes = [vp, C.c_int, dp, dp, dp, C.c_double, C.POINTER(Overrides),
                           C.POINTER(C.c_int), dp]
    L.ewg_tune_kernels.argtypes = [vp, C.c_int, dp, dp, dp, C.c_double, C.POINTER(Overrides),
                                   C.c_int, C.POINTER(KernelShape), dp]
    L.ewg_set_kernel_shape.argtypes = [vp, C.POINTER(KernelShape)]
    L.ewg_grid_memory.argtypes = [C.c_int, dp, dp, C.c_double, C.POINTER(Overrides), dp]
    L.ewg_device_memory.argtypes = [C.c_int, dp, dp, C.c_double, C.POINTER(Overrides), C.c_int,
                                    C.c_int, dp]
    L.ewg_potential_force_device.argtypes = [vp, C.c_int, vp, vp, dp, C.c_double, vp, vp,
                                             C.POINTER(Overrides)]
    L.ewg_direct_potential_force.argtypes = [vp, C.c_int, dp, dp, dp, C.c_double, dp, dp, dp, dp, dp]
    L.ewg_set_lattice.argtypes = [vp, dp]
    L.ewg_set_coords.argtypes = [vp, C.c_int, dp]
    L.ewg_set_charges.argtypes = [vp, dp]
    L.ewg_shift.argtypes = [vp, C.c_double, dp]
    L.ewg_shift_force.argtypes = [vp, C.c_double, dp, dp]
    L.ewg_shift_batch.argtypes = [vp, C.c_double, C.c_int, dp, dp]
    L.ewg_stress.argtypes = [vp, C.c_double, C.c_double, dp]
    L.ewg_stress_fast.argtypes = [vp, C.c_double, dp]
    L.ewg_xlbomd_gradients.argtypes = [vp, C.c_double, dp, dp]
    L.ewg_set_background.argtypes = [vp, C.c_int]
    L.ewg_set_force_scheme.argtypes = [vp, C.c_int]
    L.ewg_set_point_engine.argtypes = [vp, C.c_int]
    L.ewg_set_graphs.argtypes = [vp, C.c_int]
    L.ewg_potential_at.argtypes = [vp, C.c_int, dp, C.c_int, dp, dp, dp, dp, dp, C.c_double,
                                   C.c_double, dp]
    L.ewg_potential_gradient_at.argtypes = [vp, C.c_int, dp, C.c_int, dp, dp, dp, dp, C.c_double,
                                            C.c_double, dp]
    L.ewg_external_pot_grad.argtypes = [vp, C.c_int, dp, C.c_int, dp, dp, dp, C.c_int, dp, dp,
                                        C.c_double, C.c_double, dp, dp]
    L.ewg_last_stress_setup.argtypes = [vp, dp, dp, dp, ip]
    L.ewg_batch_potential_force.argtypes = [vp, C.c_int, ip, dp, dp, dp, C.c_double, dp, dp, ip]
    L.ewg_batch_potential_force_ov.argtypes = [vp, C.c_int, ip, dp, dp, dp, C.c_double, dp, dp, ip,
                                               C.POINTER(Overrides)]
    L.ewg_set_batch_lanes.argtypes = [vp, C.c_int]
    L.ewg_set_profiling.argtypes = [vp, C.c_int]
    L.ewg_stage_count.argtypes = []
    L.ewg_stage_name.argtypes = [C.c_int]
    L.ewg_stage_name.restype = C.c_char_p
    L.ewg_stage_times.argtypes = [vp, dp, C.POINTER(C.c_longlong), C.c_int]
    L.ewg_reset_stage_times.argtypes = [vp]
    L.ewg_set_stream.argtypes = [vp, vp]
    _lib = L
    return L


def status_string(code: int) -> str:
    return lib().ewg_status_string(int(code)).decode()


def _check(rc: int):
    if rc:
        raise EwaldError(rc, status_string(rc))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _overrides(alpha_in=None, r_cut_in=None, k_cut_in=None, nModes_in=None, windowCutoff_in=None):
    ov = Overrides()
    if alpha_in is not None:
        ov.has_alpha, ov.alpha = 1, float(alpha_in)
    if r_cut_in is not None:
        ov.has_r_cut, ov.r_cut = 1, float(r_cut_in)
    if k_cut_in is not None:
        ov.has_k_cut, ov.k_cut = 1, float(k_cut_in)
    if nModes_in is not None:
        ov.has_n_modes, ov.n_modes = 1, int(nModes_in)
    if windowCutoff_in is not None:
        ov.has_window_cutoff, ov.window_cutoff = 1, int(windowCutoff_in)
    return ov


def _positions_fortran(positions, n):
    pos = np.asarray(positions, dtype=np.float64)
    if pos.ndim != 2 or pos.shape[1] != 3 or pos.shape[0] < n:
        raise EwaldError(2, "ewald_fft_3d: positions must be (N,3)")
    return np.asfortranarray(pos[:n])


def _lat_fortran(latVecs):
    lat = np.asarray(latVecs, dtype=np.float64)
    if lat.shape != (3, 3):
        raise EwaldError(2, "latVecs must be (3,3)")
    return np.asfortranarray(lat)


class Context:
    """One device context (stream, device buffers, plan caches) of the library."""

    def __init__(self, device: int = 0, precision: int = FP64):
        self._h = C.c_void_p()
        _check(lib().ewg_create(C.byref(self._h), int(device), int(precision)))
        self.precision = precision

    def close(self):
        if self._h:
            lib().ewg_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    @property
    def kernel_launches(self) -> int:
        return int(lib().ewg_kernel_launches(self._h))

    def set_stream(self, stream_handle: int | None):
        """Run on a caller's CUDA stream (e.g. torch.cuda.current_stream().cuda_stream)."""
        _check(lib().ewg_set_stream(self._h, C.c_void_p(stream_handle) if stream_handle else None))

    def set_profiling(self, on: bool = True):
        _check(lib().ewg_set_profiling(self._h, 1 if on else 0))

    def stage_times(self, reset: bool = False) -> dict:
        """{stage: (milliseconds, launches)} accumulated while profiling is on."""
        L = lib()
        n = L.ewg_stage_count()
        ms = np.zeros(n)
        la = (C.c_longlong * n)()
        _check(L.ewg_stage_times(self._h, _dp(ms), la, n))
        if reset:
            _check(L.ewg_reset_stage_times(self._h))
        return {L.ewg_stage_name(i).decode(): (float(ms[i]), int(la[i])) for i in range(n)}

    def fp64_mma_peak(self) -> float:
        """Measured dense FP64 tensor-core rate of this context's GPU, TFLOP/s."""
        v = C.c_double()
        _check(lib().ewg_fp64_mma_peak(self._h, C.byref(v)))
        return float(v.value)

    def last_params(self) -> dict:
        p = Params()
        _check(lib().ewg_last_params(self._h, C.byref(p)))
        return p.as_dict()

    # -- library surface ----------------------------------------------------
    def potential_force(self, positions, charges, latVecs, tol=1e-10, want_force=True, **ov):
        q = np.ascontiguousarray(charges, dtype=np.float64)
        n = q.shape[0]
        pos = _positions_fortran(positions, n)
        lat = _lat_fortran(latVecs)
        pot = np.empty(n)
        force = np.empty((n, 3)) if want_force else None
        o = _overrides(**ov)
        _check(lib().ewg_potential_force(self._h, n, _dp(pos), _dp(q), _dp(lat), float(tol), _dp(pot),
                                         _dp(force) if want_force else None, C.byref(o)))
        return (pot, force) if want_force else pot

    def tune(self, positions, charges, latVecs, target=1e-6):
        """Fastest parameter set and force scheme of this form whose RMS
        relative force error against the FP64 i k form at tol 1e-10 is at most
        target/2 (potential: target) on this configuration.  Returns
        (overrides, scheme, report): overrides as keyword arguments for
        potential_force & co., scheme for set_force_scheme."""
        q = np.ascontiguousarray(charges, dtype=np.float64)
        n = q.shape[0]
        pos = _positions_fortran(positions, n)
        lat = _lat_fortran(latVecs)
        o = Overrides()
        scheme = C.c_int()
        rep = np.zeros(4)
        _check(lib().ewg_tune(self._h, n, _dp(pos), _dp(q), _dp(lat), float(target), C.byref(o),
                              C.byref(scheme), _dp(rep)))
        ov = dict(alpha_in=o.alpha, r_cut_in=o.r_cut, k_cut_in=o.k_cut,
                  windowCutoff_in=o.window_cutoff)
        return ov, int(scheme.value), dict(force_rms=float(rep[0]), pot_rms=float(rep[1]),
                                           ms=float(rep[2]), candidates=int(rep[3]))

    def tune_kernels(self, positions, charges, latVecs, tol=1e-10, want_force=True, **ov):
        """Kernel shapes for this configuration's bucket (precision form, force
        grids, atom octave, grid, window), searched by timing when the bucket is
        new and cached in the context; later evaluations in the bucket run
        them.  Returns (shape dict, (default ms, tuned ms)), the times 0 when the
        bucket was already tuned."""
        q = np.ascontiguousarray(charges, dtype=np.float64)
        n = q.shape[0]
        pos = _positions_fortran(positions, n)
        lat = _lat_fortran(latVecs)
        o = _overrides(**ov)
        ks = KernelShape()
        ms = np.zeros(2)
        _check(lib().ewg_tune_kernels(self._h, n, _dp(pos), _dp(q), _dp(lat), float(tol),
                                      C.byref(o), int(bool(want_force)), C.byref(ks), _dp(ms)))
        return ks.as_dict(), (float(ms[0]), float(ms[1]))

    def set_kernel_shape(self, shape=None):
        """Pin kernel shapes (a dict of KernelShape fields, 0 or missing =
        default) for every later evaluation; None returns to the tuned buckets."""
        if shape is None:
            _check(lib().ewg_set_kernel_shape(self._h, None))
            return
        ks = KernelShape(**{k: int(v) for k, v in shape.items()})
        _check(lib().ewg_set_kernel_shape(self._h, C.byref(ks)))

    def potential_force_stress(self, positions, charges, latVecs, tol=1e-10, **ov):
        """Potential, force and the NFFT-based stress sigma = (2/V) dE/d(strain)
        (3 x 3, the invRStress convention) of one evaluation."""
        q = np.ascontiguousarray(charges, dtype=np.float64)
        n = q.shape[0]
        pos = _positions_fortran(positions, n)
        lat = _lat_fortran(latVecs)
        pot = np.empty(n)
        force = np.empty((n, 3))
        sigma = np.empty((3, 3), order="F")
        o = _overrides(**ov)
        _check(lib().ewg_potential_force_stress(self._h, n, _dp(pos), _dp(q), _dp(lat), float(tol),
                                                _dp(pot), _dp(force), _dp(sigma), C.byref(o)))
        return pot, force, np.array(sigma)

    def potential_force_device(self, coords, charges, latVecs, tol, pot, force=None, **ov):
        """All of coords (N,3) atom-major, charges, pot, force (N,3) are CUDA
        tensors (float64, contiguous); only latVecs is host."""
        n = int(charges.shape[0])
        lat = _lat_fortran(latVecs)
        o = _overrides(**ov)
        _check(lib().ewg_potential_force_device(
            self._h, n, C.c_void_p(coords.data_ptr()), C.c_void_p(charges.data_ptr()), _dp(lat),
            float(tol), C.c_void_p(pot.data_ptr()),
            C.c_void_p(force.data_ptr()) if force is not None else None, C.byref(o)))

    def direct_potential_force(self, positions, charges, latVecs, tol=1e-12, want_force=True,
                               alpha_in=None, r_cut_in=None, k_cut_in=None):
        q = np.ascontiguousarray(charges, dtype=np.float64)
        n = q.shape[0]
        pos = _positions_fortran(positions, n)
        lat = _lat_fortran(latVecs)
        pot = np.empty(n)
        force = np.empty((n, 3)) if want_force else None
        opt = [C.byref(C.c_double(v)) if v is not None else None for v in (alpha_in, r_cut_in, k_cut_in)]
        _check(lib().ewg_direct_potential_force(self._h, n, _dp(pos), _dp(q), _dp(lat), float(tol),
                                                _dp(pot), _dp(force) if want_force else None, *opt))
        return (pot, force) if want_force else pot

    def direct_ground_truth(self, positions, charges, latVecs, tol=1e-13, want_force=True):
        """FP64 direct-Ewald result for error reports on large cells.

        The direct engine with its splitting pinned so that the real-space
        cutoff, sqrt(-ln tol)/alpha, is a quarter of the narrowest plane
        spacing of the cell: the real-space sum then runs over the cell list
        (only pairs beyond the cutoff are skipped) and the structure-factor sum
        over the k sphere stays small, so 216,000 atoms take about a second.
        Both truncations are at the tol level, far below the mixed form's
        errors.  Returns (pot, force) like direct_potential_force."""
        alpha = direct_ground_truth_alpha(latVecs, tol)
        return self.direct_potential_force(positions, charges, latVecs, tol, want_force,
                                           alpha_in=alpha)

    def set_batch_lanes(self, lanes: int):
        """Batched calls: 0 (default) runs every stage of all cells in one
        segmented launch; 1..16 runs the cells on that many concurrent lanes."""
        _check(lib().ewg_set_batch_lanes(self._h, int(lanes)))

    def batch_potential_force(self, cells, tol=1e-10, want_force=True, **ov):
        """cells: list of (positions (N_c,3), charges, lat_rows).  Returns lists.
        Keyword overrides (alpha_in, ...) apply to every cell."""
        offsets = np.zeros(len(cells) + 1, dtype=np.int32)
        for i, (p, q, _) in enumerate(cells):
            offsets[i + 1] = offsets[i] + len(q)
        coords = np.ascontiguousarray(np.concatenate([np.asarray(p) for p, _, _ in cells]), dtype=np.float64)
        charges = np.ascontiguousarray(np.concatenate([np.asarray(q) for _, q, _ in cells]), dtype=np.float64)
        lat = np.ascontiguousarray(np.concatenate([np.asfortranarray(np.asarray(l, dtype=np.float64)).ravel(order="F")
                                                   for _, _, l in cells]))
        total = int(offsets[-1])
        pot = np.empty(total)
        force = np.empty((total, 3)) if want_force else None
        status = np.zeros(len(cells), dtype=np.int32)
        o = _overrides(**ov)
        rc = lib().ewg_batch_potential_force_ov(
            self._h, len(cells), offsets.ctypes.data_as(C.POINTER(C.c_int)), _dp(coords), _dp(charges),
            _dp(lat), float(tol), _dp(pot), _dp(force) if want_force else None,
            status.ctypes.data_as(C.POINTER(C.c_int)), C.byref(o))
        _check(rc)
        pots = [pot[offsets[i]:offsets[i + 1]] for i in range(len(cells))]
        forces = [force[offsets[i]:offsets[i + 1]] for i in range(len(cells))] if want_force else None
        return pots, forces

    # -- TCoulomb surface ---------------------------------------------------
    def set_lattice(self, lat_cols):
        lat = np.asfortranarray(np.asarray(lat_cols, dtype=np.float64))
        _check(lib().ewg_set_lattice(self._h, _dp(lat)))

    def set_coords(self, coords_3n):
        x = np.ascontiguousarray(coords_3n, dtype=np.float64)
        _check(lib().ewg_set_coords(self._h, x.shape[0], _dp(x)))

    def set_charges(self, dq):
        q = np.ascontiguousarray(dq, dtype=np.float64)
        _check(lib().ewg_set_charges(self._h, _dp(q)))

    def shift(self, tol, n):
        out = np.empty(n)
        _check(lib().ewg_shift(self._h, float(tol), _dp(out)))
        return out

    def shift_force(self, tol, n):
        out = np.empty(n)
        f = np.empty((n, 3))
        _check(lib().ewg_shift_force(self._h, float(tol), _dp(out), _dp(f)))
        return out, f

    def shift_batch(self, tol, charges, out=None):
        """k charge updates on the resident geometry in one submission
        (ewg_shift_batch): charges (k, N) -> shifts (k, N), each row what
        set_charges(row) then shift() would give."""
        q = np.ascontiguousarray(charges, dtype=np.float64)
        if q.ndim != 2:
            raise EwaldError(2, "ewald_b200: charges must be (k, N)")
        if out is None:
            out = np.empty_like(q)
        _check(lib().ewg_shift_batch(self._h, float(tol), q.shape[0], _dp(q), _dp(out)))
        return out

    # -- potentials and gradients at arbitrary points (stock Ewald) -----------
    def potential_at(self, targets, sources, charges, lat_cols, tol_ewald=1e-9, alpha=0.0,
                     blur=None, eps_soften=None):
        """getPotential (coulomb.F90:3122-3153): (N,3) targets, (M,3) sources."""
        t = np.ascontiguousarray(targets, dtype=np.float64)
        x = np.ascontiguousarray(sources, dtype=np.float64)
        q = np.ascontiguousarray(charges, dtype=np.float64)
        lat = np.asfortranarray(np.asarray(lat_cols, dtype=np.float64))
        b = None if blur is None else np.ascontiguousarray(blur, dtype=np.float64)
        eps = None if eps_soften is None else np.array([float(eps_soften)])
        out = np.empty(t.shape[0])
        _check(lib().ewg_potential_at(self._h, t.shape[0], _dp(t), x.shape[0], _dp(x), _dp(q),
                                      _dp(b) if b is not None else None,
                                      _dp(eps) if eps is not None else None, _dp(lat),
                                      float(tol_ewald), float(alpha), _dp(out)))
        return out

    def potential_gradient_at(self, targets, sources, charges, lat_cols, tol_ewald=1e-9,
                              alpha=0.0, blur=None):
        """getPotentialGradient (coulomb.F90:3157-3194): (N,3) gradients."""
        t = np.ascontiguousarray(targets, dtype=np.float64)
        x = np.ascontiguousarray(sources, dtype=np.float64)
        q = np.ascontiguousarray(charges, dtype=np.float64)
        lat = np.asfortranarray(np.asarray(lat_cols, dtype=np.float64))
        b = None if blur is None else np.ascontiguousarray(blur, dtype=np.float64)
        out = np.empty((t.shape[0], 3))
        _check(lib().ewg_potential_gradient_at(self._h, t.shape[0], _dp(t), x.shape[0], _dp(x),
                                               _dp(q), _dp(b) if b is not None else None, _dp(lat),
                                               float(tol_ewald), float(alpha), _dp(out)))
        return out

    def external_pot_grad(self, atoms, ext, atom_charges, ext_charges, lat_cols, ham_deriv,
                          atom_grads, ext_grads, tol_ewald=1e-9, alpha=0.0, ext_blur=None):
        """addExternalPotGrad (coulomb.F90:3198-3248): adds into the (N,3) and
        (M,3) gradient arrays in place (C-contiguous float64)."""
        a = np.ascontiguousarray(atoms, dtype=np.float64)
        e = np.ascontiguousarray(ext, dtype=np.float64)
        qa = np.ascontiguousarray(atom_charges, dtype=np.float64)
        qe = np.ascontiguousarray(ext_charges, dtype=np.float64)
        lat = np.asfortranarray(np.asarray(lat_cols, dtype=np.float64))
        b = None if ext_blur is None else np.ascontiguousarray(ext_blur, dtype=np.float64)
        _check(lib().ewg_external_pot_grad(self._h, a.shape[0], _dp(a), e.shape[0], _dp(e),
                                           _dp(qa), _dp(qe), 1 if ham_deriv else 0,
                                           _dp(b) if b is not None else None, _dp(lat),
                                           float(tol_ewald), float(alpha), _dp(atom_grads),
                                           _dp(ext_grads)))
        return atom_grads, ext_grads

    def set_background(self, on: bool = True):
        """Charged cells with a uniform neutralising background (off by default)."""
        _check(lib().ewg_set_background(self._h, 1 if on else 0))

    def set_graphs(self, on: bool = True):
        """Record repeated evaluations as CUDA graphs and replay them (default on)."""
        _check(lib().ewg_set_graphs(self._h, 1 if on else 0))

    def set_point_engine(self, engine: int):
        """Engine of potential_at / potential_gradient_at / external_pot_grad:
        POINTS_AUTO (default), POINTS_STOCK or POINTS_MESH."""
        _check(lib().ewg_set_point_engine(self._h, int(engine)))

    def set_force_scheme(self, scheme: int):
        """FORCE_IK (the reference's scheme) or FORCE_AD (window derivatives)."""
        _check(lib().ewg_set_force_scheme(self._h, int(scheme)))

    def xlbomd_gradients(self, tol, dq_out):
        """Gradient (N,3) of the XLBOMD shadow energy of the resident state."""
        qo = np.ascontiguousarray(dq_out, dtype=np.float64)
        g = np.zeros((qo.shape[0], 3))
        _check(lib().ewg_xlbomd_gradients(self._h, float(tol), _dp(qo), _dp(g)))
        return g

    def stress_fast(self, tol):
        """NFFT-based stress (2/V) dE/d(strain) of the resident state."""
        s = np.empty(9)
        _check(lib().ewg_stress_fast(self._h, float(tol), _dp(s)))
        return s.reshape(3, 3, order="F")

    def stress(self, tol_ewald, alpha=0.0):
        s = np.empty(9)
        _check(lib().ewg_stress(self._h, float(tol_ewald), float(alpha), _dp(s)))
        return s.reshape(3, 3, order="F")

    def last_stress_setup(self):
        a, r, g, n = C.c_double(), C.c_double(), C.c_double(), C.c_int()
        _check(lib().ewg_last_stress_setup(self._h, C.byref(a), C.byref(r), C.byref(g), C.byref(n)))
        return {"alpha": a.value, "max_r": r.value, "max_g": g.value, "n_g": n.value}


class PackedCells:
    """A batch of cells packed once in the C ABI's host layout (CSR offsets,
    coords (3, total) atom-major, charges, 9 lattice values per cell, outputs),
    for repeated batched calls on the same cells (an MD or SCC loop over a set
    of structures): each call then passes these arrays straight to
    ewg_batch_potential_force_ov.  alloc(shape) makes the host arrays
    (np.empty by default; page-locked arrays make the call's copies faster)."""

    def __init__(self, cells, want_force=True, alloc=None):
        alloc = alloc or (lambda shape: np.empty(shape, dtype=np.float64))
        n = len(cells)
        self.offsets = np.zeros(n + 1, dtype=np.int32)
        for i, (_, q, _) in enumerate(cells):
            self.offsets[i + 1] = self.offsets[i] + len(q)
        total = int(self.offsets[-1])
        self.coords = alloc((total, 3))
        self.charges = alloc((total,))
        self.lat = alloc((n, 9))
        for i, (p, q, lat) in enumerate(cells):
            a, b = self.offsets[i], self.offsets[i + 1]
            self.coords[a:b] = np.asarray(p)
            self.charges[a:b] = np.asarray(q)
            self.lat[i] = np.asarray(lat, dtype=np.float64).ravel(order="F")
        self.pot = alloc((total,))
        self.force = alloc((total, 3)) if want_force else None
        self.status = np.zeros(n, dtype=np.int32)

    def set_charges(self, i, q):
        """New charges for cell i (same atom count)."""
        self.charges[self.offsets[i]:self.offsets[i + 1]] = q

    def evaluate(self, ctx, tol=1e-10, **ov):
        """One batched call on ctx; results in self.pot and self.force."""
        o = _overrides(**ov)
        _check(lib().ewg_batch_potential_force_ov(
            ctx.handle, len(self.status), self.offsets.ctypes.data_as(C.POINTER(C.c_int)),
            _dp(self.coords), _dp(self.charges), _dp(self.lat), float(tol), _dp(self.pot),
            _dp(self.force) if self.force is not None else None,
            self.status.ctypes.data_as(C.POINTER(C.c_int)), C.byref(o)))
        return self


_default = {}


def direct_ground_truth_alpha(latVecs, tol=1e-13) -> float:
    """Splitting of Context.direct_ground_truth: the real-space cutoff
    sqrt(-ln tol)/alpha equals a quarter of the narrowest plane spacing
    1/max|b_i| of the cell (lattice vectors as rows)."""
    lat = np.asarray(latVecs, dtype=np.float64)
    rec = np.linalg.inv(lat).T  # rows b_i with b_i . a_j = delta_ij
    spacing = 1.0 / np.max(np.linalg.norm(rec, axis=1))
    return float(np.sqrt(-np.log(tol)) / (0.25 * spacing))


def default_context(precision: int = FP64) -> Context:
    if precision not in _default:
        _default[precision] = Context(0, precision)
    return _default[precision]


# ---- reference-shaped module functions -------------------------------------

def ewald_potential_force(positions, charges, nParticle, latVecs, tol=None, pot=None, force=None,
                          alpha_in=None, r_cut_in=None, k_cut_in=None, nModes_in=None,
                          windowCutoff_in=None, context: Context | None = None):
    """ewald_potential_force (fft/ewald_fft_3d.f90:36-134).  ``pot`` (N) and the
    optional ``force`` (3, N) are filled in place; both are also returned."""
    ctx = context or default_context(FP64)
    n = int(nParticle)
    q = np.ascontiguousarray(np.asarray(charges, dtype=np.float64)[:n])
    tolerance = 1.0e-10 if tol is None else float(tol)
    if pot is not None and np.asarray(pot).shape[0] < n:
        raise EwaldError(2, "ewald_fft_3d: pot must be sized (N)")
    if force is not None and (force.shape[0] != 3 or force.shape[1] < n):
        raise EwaldError(2, "ewald_fft_3d: force must be sized (3,N)")
    res = ctx.potential_force(positions, q, latVecs, tolerance, want_force=force is not None,
                              alpha_in=alpha_in, r_cut_in=r_cut_in, k_cut_in=k_cut_in,
                              nModes_in=nModes_in, windowCutoff_in=windowCutoff_in)
    p, f = (res if force is not None else (res, None))
    if pot is None:
        pot = p
    else:
        pot[:n] = p
    if force is not None:
        force[:, :n] = f.T
    return (pot, force) if force is not None else pot


def ewald_parameters(positions, charges, nParticle, latVecs, tol=None, alpha_in=None, r_cut_in=None,
                     k_cut_in=None, nModes_in=None, windowCutoff_in=None) -> dict:
    """ewald_parameters (fft/ewald_fft_3d.f90:142-191): the parameter set."""
    n = int(nParticle)
    q = np.ascontiguousarray(np.asarray(charges, dtype=np.float64)[:n])
    lat = _lat_fortran(latVecs)
    p = Params()
    o = _overrides(alpha_in, r_cut_in, k_cut_in, nModes_in, windowCutoff_in)
    _check(lib().ewg_parameters(n, _dp(q), _dp(lat), 1.0e-10 if tol is None else float(tol),
                                C.byref(o), C.byref(p)))
    return p.as_dict()


def ewald_grid_memory(charges, nParticle, latVecs, tol=None, alpha_in=None, r_cut_in=None,
                      k_cut_in=None, nModes_in=None, windowCutoff_in=None) -> float:
    """ewald_grid_memory (fft/ewald_fft_3d.f90:197-244), in GiB."""
    n = int(nParticle)
    q = np.ascontiguousarray(np.asarray(charges, dtype=np.float64)[:n])
    lat = _lat_fortran(latVecs)
    gb = C.c_double()
    o = _overrides(alpha_in, r_cut_in, k_cut_in, nModes_in, windowCutoff_in)
    _check(lib().ewg_grid_memory(n, _dp(q), _dp(lat), 1.0e-10 if tol is None else float(tol),
                                 C.byref(o), C.byref(gb)))
    return gb.value


def ewald_direct_potential_force(positions, charges, nParticle, latVecs, tol=None, pot=None,
                                 force=None, alpha_in=None, r_cut_in=None, k_cut_in=None,
                                 context: Context | None = None):
    """ewald_potential_force of the direct engine (direct/ewald_direct_3d.f90:37-182)."""
    ctx = context or default_context(FP64)
    n = int(nParticle)
    q = np.asarray(charges, dtype=np.float64)[:n]
    res = ctx.direct_potential_force(positions, q, latVecs, 1.0e-12 if tol is None else float(tol),
                                     want_force=force is not None, alpha_in=alpha_in,
                                     r_cut_in=r_cut_in, k_cut_in=k_cut_in)
    p, f = (res if force is not None else (res, None))
    if pot is None:
        pot = p
    else:
        pot[:n] = p
    if force is not None:
        force[:, :n] = f.T
    return (pot, force) if force is not None else pot


def _env_flag(name: str) -> bool:
    return os.environ.get(name, "").strip() in ("1", "yes", "true")


class TCoulomb:
    """The periodic (pbc3d) branch of DFTB+'s TCoulomb (src/dftbp/dftb/coulomb.F90),
    with the fast engine running on the GPU.

    Call order as in hamiltonian.F90:229-233: updateLatVecs, updateCoords,
    updateCharges, updateShifts, then addShiftPerAtom / addEnergy /
    addGradients / addStress.  ``tolEwald`` is the input EwaldTolerance; values
    outside (0,1) select 1e-9 for the fast engine (coulomb.F90:348-349).
    ``DFTB_EWALD_DIRECT=1`` swaps in the direct engine at
    ``DFTB_EWALD_DIRECT_TOL`` (coulomb.F90:267-317), as the reference adapter does.
    ``fastStress=True`` (or ``DFTB_EWALD_STRESS_FAST=1``) makes addStress use the
    NFFT-based stress of the fast engine instead of the stock invRStress.
    """

    def __init__(self, nAtom: int, tolEwald: float = 1.0e-9, ewaldAlpha: float = 0.0,
                 device: int = 0, precision: int = FP64, fastStress: bool = False):
        self.nAtom = int(nAtom)
        self.fastStress = bool(fastStress) or _env_flag("DFTB_EWALD_STRESS_FAST")
        self.tolEwald = float(tolEwald)
        self.alpha = float(ewaldAlpha)
        self.ctx = Context(device, precision)
        self.latVecs = None
        self.coords = None
        self.deltaQAtom = np.zeros(self.nAtom)
        self.shiftPerAtom = np.zeros(self.nAtom)
        self.coordsUpdated = False
        self.chargesUpdated = False

    def _tol(self):
        t = self.tolEwald
        return t if 0.0 < t < 1.0 else 1.0e-9

    def _direct_tol(self):
        env = os.environ.get("DFTB_EWALD_DIRECT_TOL")
        try:
            v = float(env) if env else None
        except ValueError:
            v = None
        return v if v is not None and 0.0 < v < 1.0 else self._tol()

    def updateLatVecs(self, latVecs, recVecs=None, volume=None):
        """coulomb.F90:575-620 (latVecs with one lattice vector per column)."""
        self.latVecs = np.array(latVecs, dtype=np.float64)
        self.ctx.set_lattice(self.latVecs)
        self.coordsUpdated = False
        self.chargesUpdated = False

    def updateCoords(self, coords):
        """coulomb.F90:509-572; coords(3, N) of the central cell."""
        c = np.asarray(coords, dtype=np.float64)[:, : self.nAtom]
        self.coords = np.ascontiguousarray(c.T)
        self.ctx.set_coords(self.coords)
        self.coordsUpdated = True
        self.chargesUpdated = False

    def updateCharges(self, deltaQAtom):
        """coulomb.F90:760-781."""
        if not self.coordsUpdated:
            raise EwaldError(16, "updateCharges before updateCoords")
        self.deltaQAtom = np.array(deltaQAtom, dtype=np.float64)
        self.ctx.set_charges(self.deltaQAtom)
        self.chargesUpdated = True

    def _lat_rows(self):
        return self.latVecs.T

    def updateShifts(self):
        """coulomb.F90:786-880 with fftEwaldShift (:336-357)."""
        if not (self.coordsUpdated and self.chargesUpdated):
            raise EwaldError(16, "updateShifts before updateCoords/updateCharges")
        if _env_flag("DFTB_EWALD_DIRECT"):
            self.shiftPerAtom = self.ctx.direct_potential_force(
                self.coords, self.deltaQAtom, self._lat_rows(), self._direct_tol(), want_force=False)
        else:
            self.shiftPerAtom = self.ctx.shift(self._tol(), self.nAtom)
        return self.shiftPerAtom

    def energy(self) -> float:
        """The "Ewald energy" the adapter prints (coulomb.F90:875)."""
        return float(np.sum(self.shiftPerAtom * self.deltaQAtom) * 0.5)

    def addShiftPerAtom(self, shiftPerAtom):
        """coulomb.F90:883-898."""
        shiftPerAtom += self.shiftPerAtom
        return shiftPerAtom

    def addEnergy(self, energies, dQOutAtom=None):
        """coulomb.F90:623-653 (XLBOMD form when dQOutAtom is given)."""
        if dQOutAtom is not None:
            energies += 0.5 * self.shiftPerAtom * (2.0 * np.asarray(dQOutAtom) - self.deltaQAtom)
        else:
            energies += 0.5 * self.shiftPerAtom * self.deltaQAtom
        return energies

    def addGradients(self, gradients, dQOutAtom=None):
        """coulomb.F90:656-717 with fftEwaldAddGradients (:361-385): deriv -= F.
        With dQOutAtom, the XLBOMD shadow-energy gradient (:697-699) instead."""
        if not (self.coordsUpdated and self.chargesUpdated):
            raise EwaldError(16, "addGradients before updateCoords/updateCharges")
        if dQOutAtom is not None:
            gradients += self.ctx.xlbomd_gradients(self._tol(), dQOutAtom).T
            return gradients
        if _env_flag("DFTB_EWALD_DIRECT"):
            _, f = self.ctx.direct_potential_force(self.coords, self.deltaQAtom, self._lat_rows(),
                                                   self._direct_tol(), want_force=True)
        else:
            _, f = self.ctx.shift_force(self._tol(), self.nAtom)
        gradients -= f.T
        return gradients

    # coulomb.F90:3122-3248, periodic branch: stock Ewald between point sets with
    # this instance's lattice, tolerance and alpha (as updateLatVecs set them up).
    def getPotential(self, coords, chargeCoords, charges, blurWidths=None, epsSoften=None):
        """Potential at coords(3, N) from charges at chargeCoords(3, M)."""
        return self.ctx.potential_at(np.asarray(coords).T, np.asarray(chargeCoords).T, charges,
                                     self.latVecs, self.tolEwald, self.alpha, blur=blurWidths,
                                     eps_soften=epsSoften)

    def getPotentialGradient(self, coords, chargeCoords, charges, blurWidths=None):
        """Potential gradient (3, N) at coords(3, N)."""
        g = self.ctx.potential_gradient_at(np.asarray(coords).T, np.asarray(chargeCoords).T,
                                           charges, self.latVecs, self.tolEwald, self.alpha,
                                           blur=blurWidths)
        return g.T

    def addExternalPotGrad(self, atomCoords, extChargeCoords, atomCharges, extCharges, atomGrads,
                           extChargeGrads, tHamDeriv, extChargeBlurWidths=None):
        """Adds the derivatives into atomGrads(3, N) and extChargeGrads(3, M) in place."""
        ga = np.ascontiguousarray(np.asarray(atomGrads, dtype=np.float64).T)
        ge = np.ascontiguousarray(np.asarray(extChargeGrads, dtype=np.float64).T)
        self.ctx.external_pot_grad(np.asarray(atomCoords).T, np.asarray(extChargeCoords).T,
                                   atomCharges, extCharges, self.latVecs, tHamDeriv, ga, ge,
                                   self.tolEwald, self.alpha, ext_blur=extChargeBlurWidths)
        atomGrads[...] = ga.T
        extChargeGrads[...] = ge.T
        return atomGrads, extChargeGrads

    def addStress(self, stress):
        """coulomb.F90:721-757: stress -= 0.5 * invRStress(...)."""
        if not (self.coordsUpdated and self.chargesUpdated):
            raise EwaldError(16, "addStress before updateCoords/updateCharges")
        if self.fastStress:
            sigma = self.ctx.stress_fast(self._tol())
        else:
            sigma = self.ctx.stress(self.tolEwald, self.alpha)
        stress -= 0.5 * sigma
        return stress
