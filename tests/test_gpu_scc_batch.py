"""k SCC charge updates on the resident geometry in one submission
(ewg_shift_batch): each row equals set_charges + shift bitwise, the FP64 form
matches the oracle's fftEwaldShift (coulomb.F90:336-357) to 1e-10, and the
context's charges end as the last update's."""

import numpy as np
import pytest
from conftest import rel_max

import workloads as W

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10  # plain form vs oracle, relative to max |reference|


def updates(q, k, seed):
    return np.stack([W.charge_update(q, j, seed=seed) for j in range(k)])


@pytest.mark.parametrize("form", ["FP64", "MIXED"])
def test_batch_equals_sequential_calls_bitwise(ewald_lib, form):
    pos, q, lat = W.c2_random_4096()
    qs = updates(q, 5, seed=11)
    tol = 1e-10 if form == "FP64" else 1e-7
    seq = ewald_lib.Context(0, getattr(ewald_lib, form))
    bat = ewald_lib.Context(0, getattr(ewald_lib, form))
    try:
        for c in (seq, bat):
            c.set_lattice(lat.T)
            c.set_coords(pos)
        ref = []
        for row in qs:
            seq.set_charges(row)
            ref.append(seq.shift(tol, len(q)))
        got = bat.shift_batch(tol, qs)
        assert np.array_equal(got, np.stack(ref))
        # the resident charges are now the last update's
        assert np.array_equal(bat.shift(tol, len(q)), ref[-1])
        # a second batch on the same (now reused) geometry
        assert np.array_equal(bat.shift_batch(tol, qs[:2]), np.stack(ref[:2]))
    finally:
        seq.close()
        bat.close()


def test_batch_matches_oracle(ewald_lib, oracle):
    pos, q, lat = W.c2_random_4096()
    qs = updates(q, 3, seed=4)
    ctx = ewald_lib.Context(0, ewald_lib.FP64)
    try:
        ctx.set_lattice(lat.T)
        ctx.set_coords(pos)
        got = ctx.shift_batch(1e-10, qs)
    finally:
        ctx.close()
    for row, g in zip(qs, got):
        po = oracle.fft_potential_force(pos, row, lat, 1e-10, want_force=False)
        assert rel_max(g, po) < TOL_FP64


def test_batch_checks_every_update_first(ewald_lib):
    pos, q, lat = W.c1_small_cubic()
    ctx = ewald_lib.Context(0, ewald_lib.FP64)
    try:
        with pytest.raises(ewald_lib.EwaldError):  # before set_coords
            ctx.shift_batch(1e-10, np.stack([q]))
        ctx.set_lattice(lat.T)
        ctx.set_coords(pos)
        qs = updates(q, 3, seed=2)
        qs[2] += 0.1  # the last update is not neutral
        out = np.full_like(qs, 7.0)
        with pytest.raises(ewald_lib.EwaldError) as e:
            ctx.shift_batch(1e-10, qs, out=out)
        assert e.value.code == 3  # EWG_ERR_NOT_NEUTRAL
        assert np.all(out == 7.0)  # nothing queued, nothing written
        assert ctx.shift_batch(1e-10, np.zeros((0, len(q)))).shape == (0, len(q))
    finally:
        ctx.close()
