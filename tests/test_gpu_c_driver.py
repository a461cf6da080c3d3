"""A plain C program drives the library through include/ewald_b200.h alone.

tests/c_driver/tcoulomb_sequence.c is compiled here with gcc against the header
and linked to the in-tree libewald_b200.so; it replays DFTB+'s TCoulomb call
order (updateLatVecs, updateCoords, updateCharges + updateShifts per SCC
iteration, then addGradients and addStress; hamiltonian.F90:229-233) and one
ewald_potential_force call on the library surface.  Its outputs are compared
with the oracle (shifts, forces, the stock stress) and, for the NFFT-based
stress, which the reference does not have, with the same entry point reached
through the Python binding.  This pins the C side of the ABI that the Fortran
binding (fortran/ewald_b200.f90) binds.
"""

import os
import shutil
import subprocess

import numpy as np
import pytest
from conftest import ROOT, rel_max

import workloads as W

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10


def _build(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.fail("no C compiler to build the driver")
    libdir = os.path.join(ROOT, "dftb_fast-ewald_3d_b200")
    exe = str(tmp_path / "tcoulomb_sequence")
    subprocess.run([cc, "-std=c99", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_driver", "tcoulomb_sequence.c"), "-L", libdir,
                    "-lewald_b200", f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
    return exe


def test_c_driver_replays_tcoulomb_sequence(tmp_path, ewald_lib, oracle):
    exe = _build(tmp_path)
    pos, q, lat = W.c2_random_4096()
    n, nscc, tol, tol_ewald = len(q), 3, 1e-10, 1e-10
    rng = np.random.default_rng(7)
    dqs = []
    for it in range(nscc):
        dq = q * (1.0 + 0.1 * it) + rng.normal(0, 0.01, n)
        dqs.append(dq - dq.mean())
    inp, outp = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(inp, "wb") as f:
        np.array([n, nscc], dtype=np.int32).tofile(f)
        np.array([tol, tol_ewald], dtype=np.float64).tofile(f)
        np.ascontiguousarray(lat, dtype=np.float64).tofile(f)  # rows of lat = columns of latVecs
        np.ascontiguousarray(pos, dtype=np.float64).tofile(f)  # (N,3) rows = coords(3,N) atom-major
        np.ascontiguousarray(np.stack(dqs), dtype=np.float64).tofile(f)
    res = subprocess.run([exe, inp, outp], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    out = np.fromfile(outp, dtype=np.float64)
    o = 0

    def take(k):
        nonlocal o
        v = out[o:o + k]
        o += k
        return v

    shifts = take(nscc * n).reshape(nscc, n)
    shift_f, force = take(n), take(3 * n).reshape(n, 3)
    sigma_stock = take(9).reshape(3, 3, order="F")
    sigma_fast = take(9).reshape(3, 3, order="F")
    pot_lib, force_lib = take(n), take(3 * n).reshape(n, 3)
    assert o == out.size
    for k in range(nscc):
        po = oracle.fft_potential_force(pos, dqs[k], lat, tol, want_force=False)
        assert rel_max(shifts[k], po) < TOL_FP64
    po, fo = oracle.fft_potential_force(pos, dqs[-1], lat, tol)
    assert rel_max(shift_f, po) < TOL_FP64
    assert rel_max(force, fo) < TOL_FP64
    assert rel_max(pot_lib, po) < TOL_FP64
    assert rel_max(force_lib, fo) < TOL_FP64
    so, _ = oracle.stock_stress(pos, dqs[-1], lat.T, tol_ewald)
    assert rel_max(sigma_stock, so) < TOL_FP64
    ctx = ewald_lib.Context(0, ewald_lib.FP64)
    try:
        _, _, sf = ctx.potential_force_stress(pos, dqs[-1], lat, tol)
    finally:
        ctx.close()
    assert rel_max(sigma_fast, sf) < 1e-12
