"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE, NOT THE PRODUCT.

The oracle (``ewald_oracle.cpp``) restates the reference's fast 3D Ewald library
(src/dftbp/extlibs/fftewald) and DFTB+'s stock Ewald stress
(src/dftbp/dftb/coulomb.F90:2777-2905) on the CPU.  Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU baseline leg import this module;
the CUDA library never calls it.

parity unpinned: the reference ships no golden vectors for this path and cannot be
built in this image; see ewald_oracle.h.

Array conventions follow the reference library's Fortran interface
(fft/ewald_fft_3d.f90:36-77): ``positions`` is (N, 3) with one atom per row,
``lat_rows`` is (3, 3) with one lattice vector per row, ``force`` is returned as
(N, 3) (the Fortran (3, N) array viewed atom-major).
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libewald_oracle.so")

STATUS_NAMES = {
    0: "ok",
    1: "nParticle must be positive",
    2: "bad argument",
    3: "the cell must be charge neutral",
    4: "tol must lie in (0,1)",
    5: "cell volume too small",
    6: "alpha must be positive",
    7: "coincident charges",
    8: "cutoffs must be positive",
    9: "failure in determining optimal alpha for Ewaldsum",
    10: "failure in getMaxREwald/getMaxGEwald",
}


class OracleError(RuntimeError):
    def __init__(self, code: int, where: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(code, 'status')} ({code})")
        self.code = code


class Overrides(C.Structure):
    _fields_ = [
        ("has_alpha", C.c_int), ("has_r_cut", C.c_int), ("has_k_cut", C.c_int),
        ("has_n_modes", C.c_int), ("has_window_cutoff", C.c_int),
        ("alpha", C.c_double), ("r_cut", C.c_double), ("k_cut", C.c_double),
        ("n_modes", C.c_int), ("window_cutoff", C.c_int),
    ]


class Params(C.Structure):
    _fields_ = [("alpha", C.c_double), ("r_cut", C.c_double), ("k_cut", C.c_double),
                ("window_cutoff", C.c_int), ("n_modes", C.c_int * 3)]

    def as_dict(self):
        return {"alpha": self.alpha, "r_cut": self.r_cut, "k_cut": self.k_cut,
                "window_cutoff": self.window_cutoff, "n_modes": tuple(self.n_modes)}


_lock = threading.Lock()
_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                build()
            L = C.CDLL(LIB_PATH)
            dp = C.POINTER(C.c_double)
            L.ewo_set_threads.argtypes = [C.c_int]
            L.ewo_fft_potential_force.argtypes = [C.c_int, dp, dp, dp, C.c_double, dp, dp,
                                                  C.POINTER(Overrides)]
            L.ewo_fft_parameters.argtypes = [C.c_int, dp, dp, C.c_double, C.POINTER(Overrides),
                                             C.POINTER(Params)]
            L.ewo_fft_grid_memory.argtypes = [C.c_int, dp, dp, C.c_double, C.POINTER(Overrides), dp]
            L.ewo_direct_potential_force.argtypes = [C.c_int, dp, dp, dp, C.c_double, dp, dp,
                                                     dp, dp, dp]
            L.ewo_real_space.argtypes = [C.c_int, dp, dp, dp, C.c_double, C.c_double, dp, dp,
                                         C.POINTER(C.c_int)]
            L.ewo_stock_stress.argtypes = [C.c_int, dp, dp, dp, C.c_double, C.c_double, dp, dp,
                                           dp, dp, C.POINTER(C.c_int)]
            L.ewo_potential_at.argtypes = [C.c_int, dp, C.c_int, dp, dp, dp, dp, dp, C.c_double,
                                           C.c_double, dp]
            L.ewo_potential_gradient_at.argtypes = [C.c_int, dp, C.c_int, dp, dp, dp, dp,
                                                    C.c_double, C.c_double, dp]
            L.ewo_external_pot_grad.argtypes = [C.c_int, dp, C.c_int, dp, dp, dp, C.c_int, dp, dp,
                                                C.c_double, C.c_double, dp, dp]
            L.ewo_xlbomd_gradients.argtypes = [C.c_int, dp, dp, dp, dp, C.c_double, C.c_double,
                                               dp]
            L.ewo_fft3d.argtypes = [C.c_int, C.c_int, C.c_int, dp, C.c_int]
            L.ewo_adjoint_nfft.argtypes = [C.c_int, dp, dp, dp, dp, C.c_int, C.c_int, C.c_int,
                                           C.c_int, dp]
            L.ewo_forward_nfft.argtypes = [C.c_int, dp, dp, dp, C.c_int, C.c_int, C.c_int, C.c_int,
                                           dp, dp]
            L.ewo_next_fast_length.argtypes = [C.c_int]
            L.ewo_lambert_w0.argtypes = [C.c_double]
            L.ewo_lambert_w0.restype = C.c_double
            _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _fortran_positions(positions):
    pos = np.asarray(positions, dtype=np.float64)
    return np.asfortranarray(pos)  # positions(N,3) column-major


def _fortran_lat(lat_rows):
    return np.asfortranarray(np.asarray(lat_rows, dtype=np.float64).reshape(3, 3))


def make_overrides(alpha=None, r_cut=None, k_cut=None, n_modes=None, window_cutoff=None):
    ov = Overrides()
    if alpha is not None:
        ov.has_alpha, ov.alpha = 1, float(alpha)
    if r_cut is not None:
        ov.has_r_cut, ov.r_cut = 1, float(r_cut)
    if k_cut is not None:
        ov.has_k_cut, ov.k_cut = 1, float(k_cut)
    if n_modes is not None:
        ov.has_n_modes, ov.n_modes = 1, int(n_modes)
    if window_cutoff is not None:
        ov.has_window_cutoff, ov.window_cutoff = 1, int(window_cutoff)
    return ov


def set_threads(n: int) -> int:
    return lib().ewo_set_threads(int(n))


def fft_potential_force(positions, charges, lat_rows, tol=1e-10, want_force=True, **overrides):
    """ewald_potential_force of the fast engine (fft/ewald_fft_3d.f90:36-134)."""
    pos = _fortran_positions(positions)
    q = np.ascontiguousarray(charges, dtype=np.float64)
    n = q.shape[0]
    lat = _fortran_lat(lat_rows)
    pot = np.zeros(n)
    force = np.zeros((n, 3)) if want_force else None
    ov = make_overrides(**overrides)
    rc = lib().ewo_fft_potential_force(n, _p(pos), _p(q), _p(lat), float(tol), _p(pot),
                                       _p(force) if want_force else None, C.byref(ov))
    if rc:
        raise OracleError(rc, "ewald_fft_3d")
    return (pot, force) if want_force else pot


def fft_parameters(charges, lat_rows, tol=1e-10, **overrides):
    q = np.ascontiguousarray(charges, dtype=np.float64)
    lat = _fortran_lat(lat_rows)
    out = Params()
    ov = make_overrides(**overrides)
    rc = lib().ewo_fft_parameters(q.shape[0], _p(q), _p(lat), float(tol), C.byref(ov), C.byref(out))
    if rc:
        raise OracleError(rc, "ewald_parameters")
    return out.as_dict()


def fft_grid_memory(charges, lat_rows, tol=1e-10, **overrides):
    q = np.ascontiguousarray(charges, dtype=np.float64)
    lat = _fortran_lat(lat_rows)
    gb = C.c_double()
    ov = make_overrides(**overrides)
    rc = lib().ewo_fft_grid_memory(q.shape[0], _p(q), _p(lat), float(tol), C.byref(ov), C.byref(gb))
    if rc:
        raise OracleError(rc, "ewald_grid_memory")
    return gb.value


def direct_potential_force(positions, charges, lat_rows, tol=1e-12, want_force=True,
                           alpha=None, r_cut=None, k_cut=None):
    """ewald_potential_force of the direct engine (direct/ewald_direct_3d.f90:37-182)."""
    pos = _fortran_positions(positions)
    q = np.ascontiguousarray(charges, dtype=np.float64)
    n = q.shape[0]
    lat = _fortran_lat(lat_rows)
    pot = np.zeros(n)
    force = np.zeros((n, 3)) if want_force else None

    def opt(v):
        return C.byref(C.c_double(v)) if v is not None else None

    a, r, k = (C.c_double(v) if v is not None else None for v in (alpha, r_cut, k_cut))
    rc = lib().ewo_direct_potential_force(
        n, _p(pos), _p(q), _p(lat), float(tol), _p(pot), _p(force) if want_force else None,
        C.byref(a) if a is not None else None, C.byref(r) if r is not None else None,
        C.byref(k) if k is not None else None)
    if rc:
        raise OracleError(rc, "ewald_direct_3d")
    return (pot, force) if want_force else pot


def last_stage_seconds():
    """Wall-clock split of the last fft_potential_force: real space, spread,
    FFTs, gathers, other (deconvolution, embedding, influence weights)."""
    out = np.zeros(5)
    lib().ewo_stage_seconds(_p(out))
    return dict(zip(("real_space", "spread", "fft", "gather", "other"), map(float, out)))


def real_space(positions, charges, lat_rows, alpha, r_cut):
    pos = _fortran_positions(positions)
    q = np.ascontiguousarray(charges, dtype=np.float64)
    n = q.shape[0]
    lat = _fortran_lat(lat_rows)
    pot = np.zeros(n)
    force = np.zeros((n, 3))
    used = C.c_int()
    rc = lib().ewo_real_space(n, _p(pos), _p(q), _p(lat), float(alpha), float(r_cut), _p(pot),
                              _p(force), C.byref(used))
    if rc:
        raise OracleError(rc, "short_range_potential_force")
    return pot, force, bool(used.value)


def stock_stress(coords_3n, dq, lat_cols, tol_ewald=1e-9, alpha=0.0):
    """invRStress after updateLatVecs (coulomb.F90:575-620, :2777-2905).

    ``coords_3n`` is DFTB+'s coords(3,N) given as an (N,3) array (atom-major),
    ``lat_cols`` is DFTB+'s latVecs(3,3) with one vector per column.
    Returns (sigma(3,3), info dict)."""
    x = np.ascontiguousarray(coords_3n, dtype=np.float64)
    q = np.ascontiguousarray(dq, dtype=np.float64)
    lat = np.asfortranarray(np.asarray(lat_cols, dtype=np.float64))
    out = np.zeros(9)
    a, r, g, ng = C.c_double(), C.c_double(), C.c_double(), C.c_int()
    rc = lib().ewo_stock_stress(q.shape[0], _p(x), _p(q), _p(lat), float(tol_ewald), float(alpha),
                                _p(out), C.byref(a), C.byref(r), C.byref(g), C.byref(ng))
    if rc:
        raise OracleError(rc, "invRStress")
    return out.reshape(3, 3, order="F"), {"alpha": a.value, "max_r": r.value, "max_g": g.value,
                                          "n_g": ng.value}


def _opt(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def potential_at(targets, sources, charges, lat_cols, tol_ewald=1e-9, alpha=0.0, blur=None,
                 eps_soften=None):
    """TCoulomb%getPotential (coulomb.F90:3122-3153), periodic branch: the stock
    Ewald potential at each target from the charged sources.  Coordinates (N,3)."""
    t = np.ascontiguousarray(targets, dtype=np.float64)
    x = np.ascontiguousarray(sources, dtype=np.float64)
    q = np.ascontiguousarray(charges, dtype=np.float64)
    lat = np.asfortranarray(np.asarray(lat_cols, dtype=np.float64))
    b = _opt(blur)
    eps = None if eps_soften is None else np.array([float(eps_soften)])
    out = np.zeros(t.shape[0])
    rc = lib().ewo_potential_at(t.shape[0], _p(t), x.shape[0], _p(x), _p(q),
                                _p(b) if b is not None else None,
                                _p(eps) if eps is not None else None, _p(lat), float(tol_ewald),
                                float(alpha), _p(out))
    if rc:
        raise OracleError(rc, "getPotential")
    return out


def potential_gradient_at(targets, sources, charges, lat_cols, tol_ewald=1e-9, alpha=0.0,
                          blur=None):
    """TCoulomb%getPotentialGradient (coulomb.F90:3157-3194): (N,3) gradients."""
    t = np.ascontiguousarray(targets, dtype=np.float64)
    x = np.ascontiguousarray(sources, dtype=np.float64)
    q = np.ascontiguousarray(charges, dtype=np.float64)
    lat = np.asfortranarray(np.asarray(lat_cols, dtype=np.float64))
    b = _opt(blur)
    out = np.zeros((t.shape[0], 3))
    rc = lib().ewo_potential_gradient_at(t.shape[0], _p(t), x.shape[0], _p(x), _p(q),
                                         _p(b) if b is not None else None, _p(lat),
                                         float(tol_ewald), float(alpha), _p(out))
    if rc:
        raise OracleError(rc, "getPotentialGradient")
    return out


def external_pot_grad(atoms, ext, atom_charges, ext_charges, lat_cols, ham_deriv, tol_ewald=1e-9,
                      alpha=0.0, ext_blur=None):
    """TCoulomb%addExternalPotGrad (coulomb.F90:3198-3248) added to zero arrays:
    returns (atom gradients (N,3), external-charge gradients (M,3))."""
    a = np.ascontiguousarray(atoms, dtype=np.float64)
    e = np.ascontiguousarray(ext, dtype=np.float64)
    qa = np.ascontiguousarray(atom_charges, dtype=np.float64)
    qe = np.ascontiguousarray(ext_charges, dtype=np.float64)
    lat = np.asfortranarray(np.asarray(lat_cols, dtype=np.float64))
    b = _opt(ext_blur)
    ga = np.zeros((a.shape[0], 3))
    ge = np.zeros((e.shape[0], 3))
    rc = lib().ewo_external_pot_grad(a.shape[0], _p(a), e.shape[0], _p(e), _p(qa), _p(qe),
                                     1 if ham_deriv else 0, _p(b) if b is not None else None,
                                     _p(lat), float(tol_ewald), float(alpha), _p(ga), _p(ge))
    if rc:
        raise OracleError(rc, "addExternalPotGrad")
    return ga, ge


def xlbomd_gradients(coords_3n, dq_in, dq_out, lat_cols, tol_ewald=1e-9, alpha=0.0):
    """addInvRPrimeXlbomdPeriodic (coulomb.F90:1823-1894) added to zeros: (N,3)."""
    x = np.ascontiguousarray(coords_3n, dtype=np.float64)
    qi = np.ascontiguousarray(dq_in, dtype=np.float64)
    qo = np.ascontiguousarray(dq_out, dtype=np.float64)
    lat = np.asfortranarray(np.asarray(lat_cols, dtype=np.float64))
    out = np.zeros((qi.shape[0], 3))
    rc = lib().ewo_xlbomd_gradients(qi.shape[0], _p(x), _p(qi), _p(qo), _p(lat), float(tol_ewald),
                                    float(alpha), _p(out))
    if rc:
        raise OracleError(rc, "addInvRPrimeXlbomd")
    return out


def fft3d(data, isign):
    """Unnormalised complex 3D DFT of a Fortran-ordered (n1,n2,n3) grid."""
    arr = np.asfortranarray(np.asarray(data, dtype=np.complex128)).copy(order="F")
    n1, n2, n3 = arr.shape
    rc = lib().ewo_fft3d(n1, n2, n3, arr.ctypes.data_as(C.POINTER(C.c_double)), int(isign))
    assert rc == 0
    return arr


def adjoint_nfft(t, q, M, m):
    t = np.asarray(t, dtype=np.float64)
    t1, t2, t3 = (np.ascontiguousarray(t[:, k]) for k in range(3))
    q = np.ascontiguousarray(q, dtype=np.float64)
    out = np.zeros((M[0], M[1], M[2]), dtype=np.complex128, order="F")
    lib().ewo_adjoint_nfft(q.shape[0], _p(t1), _p(t2), _p(t3), _p(q), M[0], M[1], M[2], m,
                           out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def forward_nfft(t, fhat, m):
    t = np.asarray(t, dtype=np.float64)
    t1, t2, t3 = (np.ascontiguousarray(t[:, k]) for k in range(3))
    fh = np.asfortranarray(np.asarray(fhat, dtype=np.complex128))
    M = fh.shape
    out = np.zeros(t.shape[0], dtype=np.complex128)
    lib().ewo_forward_nfft(t.shape[0], _p(t1), _p(t2), _p(t3), M[0], M[1], M[2], m,
                           fh.ctypes.data_as(C.POINTER(C.c_double)),
                           out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def next_fast_length(n):
    return lib().ewo_next_fast_length(int(n))


def lambert_w0(x):
    return lib().ewo_lambert_w0(float(x))
