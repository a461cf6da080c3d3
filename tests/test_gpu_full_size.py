"""GPU checks at the full benchmark sizes (32,769 waters; 216,000 rock-salt
sites; all 256 batched cells).

- C3 against the oracle element by element (the oracle finishes one FP64
  evaluation in seconds on the host's cores).
- C5 against the oracle element by element too (one evaluation of the 512^3
  grid takes the oracle some tens of seconds on the host's cores), and through
  size-independent properties: the unjittered 60^3 rock salt gives every site
  the Madelung potential -M q / d (an analytic pin, M = 1.747564594633182) and
  zero force; a rigid translation of the jittered crystal leaves potentials and
  forces unchanged; the resident SCC path equals fresh evaluations of the same
  charges.
- C4: every one of the 256 cells of the batched call against the oracle.
"""

import numpy as np
import pytest
from conftest import rel_max

import workloads as W

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10


@pytest.fixture(scope="module")
def ctx(ewald_lib):
    c = ewald_lib.Context(0, ewald_lib.FP64)
    yield c
    c.close()


def test_c3_full_size_matches_oracle(ctx, oracle):
    pos, q, lat = W.c3_water_32k()
    pg, fg = ctx.potential_force(pos, q, lat, 1e-10)
    po, fo = oracle.fft_potential_force(pos, q, lat, 1e-10)
    assert rel_max(pg, po) < TOL_FP64, rel_max(pg, po)
    assert rel_max(fg, fo) < TOL_FP64, rel_max(fg, fo)


def test_c5_full_size_matches_oracle(ctx, oracle):
    pos, q, lat = W.c5_rock_salt_216k()
    pg, fg = ctx.potential_force(pos, q, lat, 1e-10)
    po, fo = oracle.fft_potential_force(pos, q, lat, 1e-10)
    assert rel_max(pg, po) < TOL_FP64, rel_max(pg, po)
    assert rel_max(fg, fo) < TOL_FP64, rel_max(fg, fo)


def test_c5_perfect_rock_salt_gives_madelung_potential(ctx):
    d = 2.82 * W.ANGSTROM_TO_BOHR
    pos, q, lat = W.perfect_rock_salt(60, d)  # 216,000 sites, the C5 lattice unjittered
    pot, force = ctx.potential_force(pos, q, lat, 1e-10)
    madelung = -pot * q * d
    assert np.max(np.abs(madelung - W.MADELUNG_NACL)) < 1e-9
    assert np.max(np.abs(force)) * d * d < 1e-8  # every site is a centre of symmetry


def test_c5_rigid_translation_invariance(ctx):
    pos, q, lat = W.c5_rock_salt_216k()
    p0, f0 = ctx.potential_force(pos, q, lat, 1e-10)
    p1, f1 = ctx.potential_force(pos + np.array([0.37, -1.11, 2.53]), q, lat, 1e-10)
    # The mesh moves under the atoms, so only the method's own error remains.
    assert rel_max(p1, p0) < 1e-9
    assert rel_max(f1, f0) < 1e-8


def test_c5_resident_scc_matches_fresh_evaluations(ewald_lib, ctx):
    pos, q, lat = W.c5_rock_salt_216k()
    n = len(q)
    tc = ewald_lib.TCoulomb(n, tolEwald=1e-10)
    tc.updateLatVecs(lat.T)
    tc.updateCoords(pos.T)
    for k in range(3):
        dq = W.c5_charge_update(q, k)
        tc.updateCharges(dq)
        shift = tc.updateShifts()
        ref = ctx.potential_force(pos, dq, lat, 1e-10, want_force=False)
        assert rel_max(shift, ref) < 1e-13


def test_c4_all_cells_match_oracle(ctx, oracle):
    cells = W.c4_batched_cells()
    pots, forces = ctx.batch_potential_force(cells, 1e-10)
    for (pos, q, lat), pg, fg in zip(cells, pots, forces):
        po, fo = oracle.fft_potential_force(pos, q, lat, 1e-10)
        assert rel_max(pg, po) < TOL_FP64
        assert rel_max(fg, fo) < TOL_FP64
