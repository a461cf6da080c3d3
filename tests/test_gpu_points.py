"""GPU potentials and gradients at arbitrary points from a set of point charges
(TCoulomb getPotential / getPotentialGradient / addExternalPotGrad, stock Ewald)
against the oracle's restatement of the reference routines, through the C ABI.
The GPU regroups the reciprocal sum through structure factors (an exact
identity), so agreement is to rounding, bounded here at 1e-11 of the largest
value."""

import numpy as np
import pytest
from conftest import rel_max

import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-11


@pytest.fixture(scope="module")
def ctx(ewald_lib):
    c = ewald_lib.Context(0, ewald_lib.FP64)
    yield c
    c.close()


def system(n_targets=40, seed=7):
    rng = np.random.default_rng(seed)
    lat = W.triclinic_lattice(13.0, 15.0, 14.0, 82.0, 99.0, 93.0) * W.ANGSTROM_TO_BOHR
    src = rng.uniform(0, 1, (300, 3)) @ lat
    q = rng.normal(0, 0.4, 300)
    tg = rng.uniform(0, 1, (n_targets, 3)) @ lat
    tg[:3] = src[:3]  # coincident points take the self term
    return src, q, lat, tg


@pytest.mark.parametrize("blur,eps", [(None, None), (0.7, None), (None, 0.3), (0.7, 0.3)])
def test_potential_at_matches_oracle(ctx, oracle, blur, eps):
    src, q, lat, tg = system()
    b = None if blur is None else np.random.default_rng(1).uniform(0.3, 1.2, len(q))
    pg = ctx.potential_at(tg, src, q, lat.T, 1e-10, blur=b, eps_soften=eps)
    po = oracle.potential_at(tg, src, q, lat.T, 1e-10, blur=b, eps_soften=eps)
    assert rel_max(pg, po) < TOL, rel_max(pg, po)


@pytest.mark.parametrize("blur", [None, 0.7])
def test_gradient_at_matches_oracle(ctx, oracle, blur):
    src, q, lat, tg = system()
    b = None if blur is None else np.full(len(q), blur)
    gg = ctx.potential_gradient_at(tg, src, q, lat.T, 1e-10, blur=b)
    go = oracle.potential_gradient_at(tg, src, q, lat.T, 1e-10, blur=b)
    assert rel_max(gg, go) < TOL, rel_max(gg, go)


@pytest.mark.parametrize("ham_deriv", [True, False])
def test_external_pot_grad_matches_oracle(ctx, oracle, ham_deriv):
    src, q, lat, tg = system(seed=9)
    qa = np.random.default_rng(2).normal(0, 0.3, len(tg))
    blur = np.full(len(q), 0.9)
    ga = np.random.default_rng(3).normal(0, 1e-3, (len(tg), 3))  # inout: added to
    ge = np.random.default_rng(4).normal(0, 1e-3, (len(q), 3))
    ga0, ge0 = ga.copy(), ge.copy()
    ctx.external_pot_grad(tg, src, qa, q, lat.T, ham_deriv, ga, ge, 1e-10, ext_blur=blur)
    da, de = oracle.external_pot_grad(tg, src, qa, q, lat.T, ham_deriv, 1e-10, ext_blur=blur)
    assert rel_max(ga - ga0, da) < TOL
    if ham_deriv:
        assert np.array_equal(ge, ge0)
    else:
        assert rel_max(ge - ge0, de) < TOL


def test_potential_at_the_atoms_matches_the_fast_path(ctx):
    """C2 size: the stock point potential at the 4096 charges themselves equals
    the fast engine's shift to within the two methods' truncation errors at
    tol 1e-10 (a few 1e-9 of the largest potential here)."""
    pos, q, lat = W.c2_random_4096()
    ps = ctx.potential_at(pos, pos, q, lat.T, 1e-10)
    pf = ctx.potential_force(pos, q, lat, 1e-10, want_force=False)
    assert rel_max(ps, pf) < 2e-8


def test_tcoulomb_point_methods(ewald_lib, oracle):
    """The TCoulomb mirror's getPotential / getPotentialGradient / addExternalPotGrad
    use the instance's lattice, tolerance and alpha (DFTB+'s column layouts)."""
    src, q, lat, tg = system(seed=11)
    tc = ewald_lib.TCoulomb(len(q), tolEwald=1e-10)
    tc.updateLatVecs(lat.T)
    pot = tc.getPotential(tg.T, src.T, q, epsSoften=0.2)
    assert rel_max(pot, oracle.potential_at(tg, src, q, lat.T, 1e-10, eps_soften=0.2)) < TOL
    grad = tc.getPotentialGradient(tg.T, src.T, q)
    assert rel_max(grad.T, oracle.potential_gradient_at(tg, src, q, lat.T, 1e-10)) < TOL
    qa = np.linspace(-0.5, 0.5, len(tg))
    ga = np.zeros((3, len(tg)))
    ge = np.zeros((3, len(q)))
    tc.addExternalPotGrad(tg.T, src.T, qa, q, ga, ge, False)
    da, de = oracle.external_pot_grad(tg, src, qa, q, lat.T, False, 1e-10)
    assert rel_max(ga.T, da) < TOL
    assert rel_max(ge.T, de) < TOL
