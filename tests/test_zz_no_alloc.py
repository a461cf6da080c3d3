"""The allocation-free direct engine, ewg_direct_potential_force_static.

Some callers cannot allocate device memory once a run is under way, for
example a host program that gives all device memory to its own pool allocator
at start-up.  For them the library offers one entry point that takes all of its
working memory from a fixed array in device memory.  These tests call it
through the C ABI on device arrays the test owns.  Over two consecutive calls
on different systems, its potential and force must match those of the regular
direct engine (ewg_direct_potential_force) within the parity tolerance the
other GPU tests use.  The array keeps the previous call's contents, so the
second call checks that nothing stale leaks into its result.  A system too large
for the array must be refused with EWG_ERR_SCRATCH_LIMIT.

This file is named to be collected last, so a run that stops at the first
failure has already run every other test.
"""

import ctypes as C

import numpy as np
import pytest
from conftest import rel_max

import workloads as W

pytestmark = pytest.mark.gpu

TOL_REL = 1e-10  # same bar as the FP64 parity tests
EWG_ERR_SCRATCH_LIMIT = 17


def _static_entry(ewald_lib):
    fn = ewald_lib.lib().ewg_direct_potential_force_static
    dp = C.POINTER(C.c_double)
    fn.argtypes = [C.c_int, C.c_void_p, C.c_void_p, dp, C.c_double, C.c_void_p, C.c_void_p, dp, dp,
                   dp, C.c_void_p]
    fn.restype = C.c_int
    return fn


def _call_static(ewald_lib, pos, q, lat, tol, want_force=True):
    import torch

    fn = _static_entry(ewald_lib)
    x = torch.tensor(np.asarray(pos), dtype=torch.float64, device="cuda").contiguous()
    qq = torch.tensor(np.asarray(q), dtype=torch.float64, device="cuda").contiguous()
    pot = torch.empty(len(q), dtype=torch.float64, device="cuda")
    force = torch.empty((len(q), 3), dtype=torch.float64, device="cuda") if want_force else None
    lat_f = np.asfortranarray(np.asarray(lat, dtype=np.float64))
    torch.cuda.synchronize()
    rc = fn(len(q), x.data_ptr(), qq.data_ptr(), lat_f.ctypes.data_as(C.POINTER(C.c_double)),
            float(tol), pot.data_ptr(), force.data_ptr() if want_force else None, None, None, None,
            None)
    torch.cuda.synchronize()
    return rc, pot.cpu().numpy(), force.cpu().numpy() if want_force else None


def _triclinic(seed, n):
    rng = np.random.default_rng(seed)
    lat = W.triclinic_lattice(13.0, 15.0, 14.0, 82.0, 99.0, 93.0) * W.ANGSTROM_TO_BOHR
    pos = rng.uniform(0, 1, size=(n, 3)) @ lat
    q = rng.normal(0, 0.4, n)
    return pos, q - q.mean(), lat


def test_static_matches_regular_direct_engine_on_two_calls(ewald_lib):
    systems = [_triclinic(31, 300), W.c1_small_cubic()]
    ctx = ewald_lib.Context(0, ewald_lib.FP64)
    try:
        for pos, q, lat in systems:  # two calls in a row on the shared scratch
            rc, pot, force = _call_static(ewald_lib, pos, q, lat, 1e-12)
            assert rc == 0, ewald_lib.status_string(rc)
            ref_pot, ref_force = ctx.direct_potential_force(pos, q, lat, 1e-12)
            assert rel_max(pot, ref_pot) < TOL_REL
            assert rel_max(force, ref_force) < TOL_REL
    finally:
        ctx.close()


def test_static_potential_only_matches_regular_direct_engine(ewald_lib):
    # Without a force array the call takes its force workspace from the fixed
    # array too; the potential must not change.
    pos, q, lat = _triclinic(32, 500)
    ctx = ewald_lib.Context(0, ewald_lib.FP64)
    try:
        for _ in range(2):
            rc, pot, _ = _call_static(ewald_lib, pos, q, lat, 1e-12, want_force=False)
            assert rc == 0, ewald_lib.status_string(rc)
            ref_pot, _ = ctx.direct_potential_force(pos, q, lat, 1e-12)
            assert rel_max(pot, ref_pot) < TOL_REL
    finally:
        ctx.close()


def test_static_refuses_oversized_systems(ewald_lib):
    pos, q, lat = W.random_cubic(400000, 160.0, 3, "normal", 0.3)
    rc, _, _ = _call_static(ewald_lib, pos, q, lat, 1e-8)
    assert rc == EWG_ERR_SCRATCH_LIMIT
    assert "scratch" in ewald_lib.status_string(rc)
