"""Charged cells (ewg_set_background): a net charge with the uniform
neutralising background of the stock Ewald engine.  Pinned against the oracle's
restatement of the stock pair sum (getPotential with the atoms as targets and
sources, whose pair function carries -pi/(V alpha^2) per unit charge) and the
stock gradient: potentials and forces agree to the two methods' truncation
errors.  Without the mode the fast path refuses the cell, as the reference's
does."""

import numpy as np
import pytest
from conftest import rel_max

import workloads as W

pytestmark = pytest.mark.gpu


def charged(gen, extra=0.05):
    pos, q, lat = gen()
    return pos, q + extra, lat


@pytest.mark.parametrize("gen", [W.c1_small_cubic, W.c2_random_4096], ids=["c1", "c2"])
def test_charged_cell_matches_stock_sum(ewald_lib, oracle, gen):
    pos, q, lat = charged(gen)
    if len(q) > 1000:
        pos, q = pos[:800], q[:800]
    ctx = ewald_lib.Context(0, ewald_lib.FP64)
    try:
        with pytest.raises(ewald_lib.EwaldError) as ei:
            ctx.potential_force(pos, q, lat, 1e-10)
        assert ei.value.code == 3
        ctx.set_background(True)
        pg, fg = ctx.potential_force(pos, q, lat, 1e-10)
    finally:
        ctx.close()
    po = oracle.potential_at(pos, pos, q, lat.T, 1e-10)
    go = oracle.potential_gradient_at(pos, pos, q, lat.T, 1e-10)
    assert rel_max(pg, po) < 2e-8, rel_max(pg, po)
    assert rel_max(fg, -q[:, None] * go) < 2e-8
