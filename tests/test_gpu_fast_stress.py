"""The NFFT-based stress of ewg_potential_force_stress (the fast path's stress,
which the reference lists as its next step and does not implement).

Pins:
- Strain derivative: with the method's parameters held fixed (alpha, cutoffs,
  modes, window), sigma = (2/V) dE/d(strain) must match central differences of
  the library's own energy E = 1/2 sum q pot under homogeneous strain of the cell
  and the positions.
- Stock stress: the reference's invRStress (restated by the oracle, and by the
  library's stock engine at full size) approximates
  the same exact Ewald stress with its own alpha and G-vector sum; both must
  agree to well within the tolerance's reach.
- The potential and force of the same call equal ewg_potential_force's.
"""

import numpy as np
import pytest
from conftest import rel_max

import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(ewald_lib):
    c = ewald_lib.Context(0, ewald_lib.FP64)
    yield c
    c.close()


def triclinic_system(n=300, seed=11):
    rng = np.random.default_rng(seed)
    lat = W.triclinic_lattice(14.0, 16.0, 15.0, 80.0, 100.0, 95.0) * W.ANGSTROM_TO_BOHR
    pos = rng.uniform(0, 1, size=(n, 3)) @ lat
    q = rng.normal(0, 0.5, n)
    return pos, q - q.mean(), lat


def strained(pos, lat, eps):
    t = np.eye(3) + eps
    return pos @ t.T, lat @ t.T


def fixed_overrides(oracle, q, lat, tol):
    p = oracle.fft_parameters(q, lat, tol)
    return {"alpha_in": p["alpha"], "r_cut_in": p["r_cut"], "nModes_in": max(p["n_modes"]),
            "windowCutoff_in": p["window_cutoff"]}


def test_stress_is_the_strain_derivative_of_the_energy(ctx, oracle):
    pos, q, lat = triclinic_system()
    ov = fixed_overrides(oracle, q, lat, 1e-10)
    _, _, sigma = ctx.potential_force_stress(pos, q, lat, 1e-10, **ov)
    V = abs(np.linalg.det(lat))
    h = 1e-5
    fd = np.zeros((3, 3))
    for a in range(3):
        for b in range(a, 3):
            e = np.zeros((3, 3))
            e[a, b] += 0.5 * h
            e[b, a] += 0.5 * h
            ener = []
            for sgn in (1.0, -1.0):
                p_s, l_s = strained(pos, lat, sgn * e)
                pot = ctx.potential_force(p_s, q, l_s, 1e-10, want_force=False, **ov)
                ener.append(0.5 * np.dot(q, pot))
            fd[a, b] = fd[b, a] = (2.0 / V) * (ener[0] - ener[1]) / (2 * h)
    assert np.allclose(sigma, sigma.T, rtol=0, atol=1e-14 * np.abs(sigma).max())
    assert rel_max(sigma, fd) < 1e-7, (sigma, fd)


def test_fast_stress_matches_stock_stress(ctx, oracle):
    pos, q, lat = triclinic_system(seed=12)
    _, _, sigma = ctx.potential_force_stress(pos, q, lat, 1e-10)
    stock, _ = oracle.stock_stress(pos, q, lat.T, 1e-10)
    # Two methods with independent truncation errors of order tol times the
    # energy scale: for this small cell that is ~1e-10 absolute, 1e-6 of max|sigma|.
    assert rel_max(sigma, stock) < 1e-5, (sigma, stock)


def test_stress_call_returns_the_same_potential_and_force(ctx):
    pos, q, lat = W.c2_random_4096()
    p0, f0 = ctx.potential_force(pos, q, lat, 1e-10)
    p1, f1, _ = ctx.potential_force_stress(pos, q, lat, 1e-10)
    assert np.array_equal(p0, p1)
    assert np.array_equal(f0, f1)


def test_c3_fast_stress_matches_stock_stress(ctx):
    """Full size: against the library's own stock engine (parity-tested against
    the oracle on smaller systems; the oracle's stock path takes minutes here)."""
    pos, q, lat = W.c3_water_32k()
    _, _, sigma = ctx.potential_force_stress(pos, q, lat, 1e-10)
    ctx.set_lattice(lat.T)
    ctx.set_coords(pos)
    ctx.set_charges(q)
    stock = ctx.stress(1e-10)
    assert rel_max(sigma, stock) < 1e-7, (sigma, stock)


def test_tcoulomb_fast_stress_sequence(ewald_lib, ctx):
    """The resident TCoulomb path (addStress with fastStress) equals the one-shot call."""
    pos, q, lat = W.c2_random_4096()
    n = len(q)
    tc = ewald_lib.TCoulomb(n, tolEwald=1e-10, fastStress=True)
    tc.updateLatVecs(lat.T)
    tc.updateCoords(pos.T)
    tc.updateCharges(q)
    tc.updateShifts()
    stress = np.zeros((3, 3))
    tc.addStress(stress)
    _, _, sigma = ctx.potential_force_stress(pos, q, lat, 1e-10)
    assert rel_max(stress, -0.5 * sigma) < 1e-12
