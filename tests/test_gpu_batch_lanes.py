"""Batched calls on concurrent lanes (ewg_set_batch_lanes): the cells give
bitwise the results of one lane (the same kernels on the same inputs, only
scheduled side by side), with and without overrides, in both precision forms,
and each lane count matches the oracle."""

import numpy as np
import pytest
from conftest import rel_max

import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_lanes_match_one_lane(ewald_lib, precision):
    cells = W.c4_batched_cells(24)
    ctx = ewald_lib.Context(0, getattr(ewald_lib, precision))
    try:
        ctx.set_batch_lanes(1)
        p1, f1 = ctx.batch_potential_force(cells, 1e-10)
        for lanes in (2, 4, 7):
            ctx.set_batch_lanes(lanes)
            for _ in range(2):  # the second call replays the lanes' recorded graphs
                pl, fl = ctx.batch_potential_force(cells, 1e-10)
                for a, b in zip(pl, p1):
                    assert np.array_equal(a, b)
                for a, b in zip(fl, f1):
                    assert np.array_equal(a, b)
    finally:
        ctx.close()


def test_lanes_with_overrides_and_oracle(ewald_lib, oracle):
    cells = [W.water_box(455, seed=3 + k) for k in range(6)]
    ctx = ewald_lib.Context(0, ewald_lib.FP64)
    try:
        ov = dict(r_cut_in=14.0, windowCutoff_in=12)
        pots, forces = ctx.batch_potential_force(cells, 1e-10, **ov)
        for (pos, q, lat), pg, fg in zip(cells, pots, forces):
            po, fo = oracle.fft_potential_force(pos, q, lat, 1e-10, r_cut=14.0, window_cutoff=12)
            assert rel_max(pg, po) < 1e-10
            assert rel_max(fg, fo) < 1e-10
    finally:
        ctx.close()


def test_lane_count_range(ewald_lib):
    ctx = ewald_lib.Context(0, ewald_lib.FP64)
    try:
        for bad in (-1, 17):
            with pytest.raises(ewald_lib.EwaldError) as e:
                ctx.set_batch_lanes(bad)
            assert e.value.code == 2  # EWG_ERR_ARG
    finally:
        ctx.close()
