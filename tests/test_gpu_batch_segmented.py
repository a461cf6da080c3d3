"""Segmented batched calls (the default, ewg_set_batch_lanes(0)): every stage
of every cell of the batch in one launch, the cells' parameters read from a
device table.  Each cell goes through the same kernels in the same order as a
cell evaluated alone, so the results are bitwise those of the one-lane path,
in both precision forms and force schemes, with and without forces, on the
first call and on the graph replays that follow; and they match the oracle.
"""

import numpy as np
import pytest
from conftest import rel_max

import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
@pytest.mark.parametrize("scheme", ["ik", "ad"])
def test_segmented_equals_one_lane_bitwise(ewald_lib, precision, scheme):
    cells = W.c4_batched_cells(20, seed=9)
    ctx = ewald_lib.Context(0, getattr(ewald_lib, precision))
    try:
        ctx.set_force_scheme(ewald_lib.FORCE_IK if scheme == "ik" else ewald_lib.FORCE_AD)
        tol = 1e-10 if precision == "FP64" else 1e-7
        ctx.set_batch_lanes(1)
        p1, f1 = ctx.batch_potential_force(cells, tol)
        q1, _ = ctx.batch_potential_force(cells, tol, want_force=False)
        ctx.set_batch_lanes(0)
        for _ in range(3):  # direct, recorded, replayed
            ps, fs = ctx.batch_potential_force(cells, tol)
            for a, b in zip(ps, p1):
                assert np.array_equal(a, b)
            for a, b in zip(fs, f1):
                assert np.array_equal(a, b)
        qs, _ = ctx.batch_potential_force(cells, tol, want_force=False)
        for a, b in zip(qs, q1):
            assert np.array_equal(a, b)
    finally:
        ctx.close()


def test_segmented_large_cells_match_oracle(ewald_lib, oracle):
    cells = [W.water_box(1365, seed=20 + k) for k in range(3)] + W.c4_batched_cells(5, seed=2)
    ctx = ewald_lib.Context(0, ewald_lib.FP64)
    try:
        pots, forces = ctx.batch_potential_force(cells, 1e-10)
        for (pos, q, lat), pg, fg in zip(cells, pots, forces):
            po, fo = oracle.fft_potential_force(pos, q, lat, 1e-10)
            assert rel_max(pg, po) < 1e-10
            assert rel_max(fg, fo) < 1e-10
    finally:
        ctx.close()
