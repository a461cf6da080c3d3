"""The mesh engine of the potentials and gradients at arbitrary points
(ewg_set_point_engine(EWG_POINTS_MESH)): the periodic pair function of
TCoulomb getPotential / getPotentialGradient / addExternalPotGrad
(dftb/coulomb.F90:3122-3248) through the NFFT and a cell list, at a cost
linear in the number of points.

The pair function is a full periodic Ewald sum and does not depend on the
splitting, so the mesh engine (its own alpha, from the fast path's chain) and
the oracle's restatement of the stock sum (DFTB+'s alpha) agree to the
truncation of either at tol 1e-10: bounded here at 1e-8 of the largest value.
A softened call keeps the stock splitting (the softening is defined on it).
At 32,769 points the mesh potential at the charges themselves equals the fast
path's shift, and four times the points cost far less than sixteen times the
time (the stock sum is quadratic).
"""

import time

import numpy as np
import pytest
from conftest import rel_max

import workloads as W

pytestmark = pytest.mark.gpu

TOL_MESH = 1e-8


@pytest.fixture(scope="module")
def ctx(ewald_lib):
    c = ewald_lib.Context(0, ewald_lib.FP64)
    c.set_point_engine(ewald_lib.POINTS_MESH)
    yield c
    c.close()


def system(n_targets=40, seed=7, n_sources=300):
    rng = np.random.default_rng(seed)
    lat = W.triclinic_lattice(13.0, 15.0, 14.0, 82.0, 99.0, 93.0) * W.ANGSTROM_TO_BOHR
    src = rng.uniform(0, 1, (n_sources, 3)) @ lat
    q = rng.normal(0, 0.4, n_sources)
    tg = rng.uniform(0, 1, (n_targets, 3)) @ lat
    tg[:3] = src[:3]  # coincident points take the self term
    return src, q, lat, tg


@pytest.mark.parametrize("blur", [None, "uniform", "per_source"])
def test_mesh_potential_at_matches_oracle(ctx, oracle, blur):
    src, q, lat, tg = system()
    b = {None: None, "uniform": np.full(len(q), 0.7),
         "per_source": np.random.default_rng(1).uniform(0.3, 1.2, len(q))}[blur]
    pg = ctx.potential_at(tg, src, q, lat.T, 1e-10, blur=b)
    po = oracle.potential_at(tg, src, q, lat.T, 1e-10, blur=b)
    assert rel_max(pg, po) < TOL_MESH, rel_max(pg, po)


def test_mesh_potential_of_a_charged_source_set(ctx, oracle):
    # A net charge: both carry the -pi Q / (V alpha^2) background with their own alpha.
    src, q, lat, tg = system(seed=3)
    q = q + 0.05
    pg = ctx.potential_at(tg, src, q, lat.T, 1e-10)
    po = oracle.potential_at(tg, src, q, lat.T, 1e-10)
    assert rel_max(pg, po) < TOL_MESH, rel_max(pg, po)


@pytest.mark.parametrize("blur", [None, 0.7])
def test_mesh_gradient_at_matches_oracle(ctx, oracle, blur):
    src, q, lat, tg = system()
    b = None if blur is None else np.full(len(q), blur)
    gg = ctx.potential_gradient_at(tg, src, q, lat.T, 1e-10, blur=b)
    go = oracle.potential_gradient_at(tg, src, q, lat.T, 1e-10, blur=b)
    assert rel_max(gg, go) < TOL_MESH, rel_max(gg, go)


@pytest.mark.parametrize("ham_deriv", [True, False])
def test_mesh_external_pot_grad_matches_oracle(ctx, oracle, ham_deriv):
    src, q, lat, tg = system(seed=9)
    qa = np.random.default_rng(2).normal(0, 0.3, len(tg))
    blur = np.full(len(q), 0.9)
    ga = np.random.default_rng(3).normal(0, 1e-3, (len(tg), 3))
    ge = np.random.default_rng(4).normal(0, 1e-3, (len(q), 3))
    ga0, ge0 = ga.copy(), ge.copy()
    ctx.external_pot_grad(tg, src, qa, q, lat.T, ham_deriv, ga, ge, 1e-10, ext_blur=blur)
    da, de = oracle.external_pot_grad(tg, src, qa, q, lat.T, ham_deriv, 1e-10, ext_blur=blur)
    assert rel_max(ga - ga0, da) < TOL_MESH
    if ham_deriv:
        assert np.array_equal(ge, ge0)
    else:
        assert rel_max(ge - ge0, de) < TOL_MESH


def test_softened_call_keeps_the_stock_sum(ewald_lib, ctx):
    src, q, lat, tg = system(seed=5)
    stock = ewald_lib.Context(0, ewald_lib.FP64)
    try:
        stock.set_point_engine(ewald_lib.POINTS_STOCK)
        ps = stock.potential_at(tg, src, q, lat.T, 1e-10, eps_soften=0.3)
    finally:
        stock.close()
    pm = ctx.potential_at(tg, src, q, lat.T, 1e-10, eps_soften=0.3)
    assert np.array_equal(pm, ps)


def test_mesh_potential_at_the_charges_equals_the_fast_path_at_32k(ewald_lib, ctx):
    pos, q, lat = W.c3_water_32k()
    pm = ctx.potential_at(pos, pos, q, lat.T, 1e-10)
    pf = ewald_lib.Context(0, ewald_lib.FP64)
    try:
        ref = pf.potential_force(pos, q, lat, 1e-10, want_force=False)
    finally:
        pf.close()
    assert rel_max(pm, ref) < TOL_MESH, rel_max(pm, ref)


def test_mesh_cost_is_linear_in_the_points(ctx):
    def timed(n_mol):
        # best of several calls: a host or allocation hiccup in one call must
        # not decide the comparison
        pos, q, lat = W.water_box(n_mol, seed=17)
        ctx.potential_at(pos, pos, q, lat.T, 1e-10)  # first call: buffers and plans
        best = float("inf")
        for _ in range(7):
            t0 = time.perf_counter()
            ctx.potential_at(pos, pos, q, lat.T, 1e-10)
            best = min(best, time.perf_counter() - t0)
        return best

    t_small = timed(2731)   # 8,193 points on 8,193 charges
    t_large = timed(10923)  # 32,769 on 32,769: four times the points
    assert t_large < 8.0 * t_small, (t_small, t_large)
    assert t_large < 1.0, t_large
