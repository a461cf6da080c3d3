"""XLBOMD gradients (TCoulomb addGradients with dQOutAtom; the reference's
addInvRPrimeXlbomdPeriodic, coulomb.F90:1823-1894).

The library takes the fast path's gradient of E(qi + qo) - E(qo) - 2 E(qi)
(three evaluations, one parameter set); the oracle restates the reference's
stock-Ewald pair sum.  The two methods carry independent truncation errors at
the tolerance, so they agree to ~1e-9 of the largest gradient; with qo = qi the
shadow energy is the ordinary energy and the gradient must equal -force to
rounding."""

import numpy as np
import pytest
from conftest import rel_max

import workloads as W

pytestmark = pytest.mark.gpu


def charges_out(q, seed=1, scale=0.05):
    rng = np.random.default_rng(seed)
    qo = q + rng.normal(0, scale, len(q))
    return qo - qo.mean()


@pytest.mark.parametrize("gen", [W.c1_small_cubic, W.c2_random_4096], ids=["c1", "c2"])
def test_xlbomd_matches_oracle(ewald_lib, oracle, gen):
    pos, q, lat = gen()
    if len(q) > 1000:  # the oracle's pair sum is O(N^2 nG): a neutral subset
        pos, q = pos[:600], q[:600] - q[:600].mean()
    qo = charges_out(q)
    tc = ewald_lib.TCoulomb(len(q), tolEwald=1e-10)
    tc.updateLatVecs(lat.T)
    tc.updateCoords(pos.T)
    tc.updateCharges(q)
    grad = np.zeros((3, len(q)))
    tc.addGradients(grad, dQOutAtom=qo)
    ref = oracle.xlbomd_gradients(pos, q, qo, lat.T, 1e-10)
    assert rel_max(grad.T, ref) < 1e-8, rel_max(grad.T, ref)


def test_xlbomd_with_equal_charges_is_the_ordinary_gradient(ewald_lib):
    pos, q, lat = W.c2_random_4096()
    tc = ewald_lib.TCoulomb(len(q), tolEwald=1e-10)
    tc.updateLatVecs(lat.T)
    tc.updateCoords(pos.T)
    tc.updateCharges(q)
    g_xl = np.zeros((3, len(q)))
    tc.addGradients(g_xl, dQOutAtom=q)
    g = np.zeros((3, len(q)))
    tc.addGradients(g)
    assert rel_max(g_xl, g) < 1e-12
