"""Pins of the CPU oracle (no GPU): the oracle must be right before the CUDA
library is checked against it.  The reference ships no golden vectors for this
path, so the oracle is pinned against numpy's FFT, an independent numpy
restatement, the direct engine, the rock-salt Madelung constant, finite
differences and the reference's own parameter values quoted for the benchmark
configurations."""

import math

import numpy as np
import pytest
from conftest import rel_max, rel_rms

import workloads as W


def test_fft_matches_numpy(oracle):
    rng = np.random.default_rng(0)
    for shp in [(6, 10, 14), (8, 9, 7), (36, 4, 5), (22, 3, 1), (2, 2, 2)]:
        a = rng.normal(size=shp) + 1j * rng.normal(size=shp)
        assert rel_max(oracle.fft3d(a, -1), np.fft.fftn(a)) < 1e-14
        assert rel_max(oracle.fft3d(a, 1), np.fft.ifftn(a) * a.size) < 1e-14


def test_next_fast_length_and_lambert(oracle):
    from scipy.special import lambertw

    # Smallest even 2,3,5,7-smooth length >= n (nfft/fft_backend.f90:73-91).
    assert [oracle.next_fast_length(n) for n in (1, 2, 3, 11, 13, 22, 34, 37, 142, 281)] == \
        [2, 2, 4, 12, 14, 24, 36, 40, 144, 288]
    for x in (1e-6, 0.3, 1.0, 10.0, 1e5, 1e12):
        assert abs(oracle.lambert_w0(x) - lambertw(x).real) <= 1e-14 * max(1.0, lambertw(x).real)
    assert oracle.lambert_w0(0.0) == 0.0


# Mode counts and window half-widths the reference chain gives for the
# benchmark configurations (fft/ewald_fft_3d_parameters.f90:52-142).
CHAIN_PINS = [
    ("c1", W.c1_small_cubic, 1e-10, (18, 18, 18), 12),
    ("c2", W.c2_random_4096, 1e-10, (64, 64, 64), 12),
    ("c3", W.c3_water_32k, 1e-10, (140, 140, 140), 12),
    ("c3_1e-9", W.c3_water_32k, 1e-9, (120, 120, 120), 11),
    ("c3_1e-6", W.c3_water_32k, 1e-6, (80, 80, 80), 8),
    ("c5", W.c5_rock_salt_216k, 1e-10, (256, 256, 256), 12),
]


@pytest.mark.parametrize("name,gen,tol,modes,m", CHAIN_PINS, ids=[c[0] for c in CHAIN_PINS])
def test_parameter_chain_pins(oracle, name, gen, tol, modes, m):
    pos, q, lat = gen()
    p = oracle.fft_parameters(q, lat, tol)
    assert p["n_modes"] == modes
    assert p["window_cutoff"] == m
    # r_cut = 3 (V/N)^(1/3) unless capped for the cell list.
    V = abs(np.linalg.det(lat))
    assert p["r_cut"] == pytest.approx(min(3.0 * (V / len(q)) ** (1 / 3), 0.999 / (3 * (1 / lat[0, 0])))
                                       if 0.999 / (3 / lat[0, 0]) >= 1.5 * (V / len(q)) ** (1 / 3)
                                       else 3.0 * (V / len(q)) ** (1 / 3), rel=1e-14)


def test_adjoint_nfft_matches_structure_factors(oracle):
    rng = np.random.default_rng(1)
    t = rng.uniform(-0.3, 1.3, size=(30, 3))
    q = rng.normal(size=30)
    M = (8, 10, 6)
    shat = oracle.adjoint_nfft(t, q, M, 12)
    ks = [np.array([a - Md if a >= Md // 2 else a for a in range(Md)]) for Md in M]
    K = np.stack(np.meshgrid(*ks, indexing="ij"), -1)
    exact = np.einsum("j,abcj->abc", q, np.exp(2j * np.pi * np.einsum("abcd,jd->abcj", K, t)))
    assert rel_max(shat, exact) < 1e-10


def test_forward_nfft_matches_direct_evaluation(oracle):
    rng = np.random.default_rng(2)
    t = rng.uniform(0, 1, size=(25, 3))
    M = (6, 8, 10)
    fh = rng.normal(size=M) + 1j * rng.normal(size=M)
    f = oracle.forward_nfft(t, fh, 12)
    ks = [np.array([a - Md if a >= Md // 2 else a for a in range(Md)]) for Md in M]
    K = np.stack(np.meshgrid(*ks, indexing="ij"), -1)
    exact = np.einsum("abc,jabc->j", fh, np.exp(-2j * np.pi * np.einsum("abcd,jd->jabc", K, t)))
    assert rel_max(f, exact) < 1e-10


def test_oracle_matches_numpy_restatement(oracle):
    import numpy_reference as npr

    rng = np.random.default_rng(7)
    lat = np.array([[9.0, 0.0, 0.0], [1.5, 8.0, 0.0], [-0.7, 1.1, 10.0]])
    n = 24
    pos = rng.uniform(0, 1, size=(n, 3)) @ lat
    q = rng.normal(size=n)
    q -= q.mean()
    kw = dict(alpha=0.45, r_cut=6.0, n_modes=10, window_cutoff=5)
    pot, force = oracle.fft_potential_force(pos, q, lat, 1e-8, **kw)
    p2, f2 = npr.potential_force(pos, q, lat, 0.45, 6.0, (10, 10, 10), 5)
    assert rel_max(pot, p2) < 1e-12
    assert rel_max(force, f2) < 1e-12


def test_fast_engine_agrees_with_direct_engine(oracle):
    for gen in (W.c1_small_cubic, W.reference_pair_fixture):
        pos, q, lat = gen()
        pf, ff = oracle.fft_potential_force(pos, q, lat, 1e-10)
        pd, fd = oracle.direct_potential_force(pos, q, lat, 1e-12)
        assert rel_max(pf, pd) < 2e-9
        assert rel_max(ff, fd) < 2e-9


def test_triclinic_fast_vs_direct(oracle):
    cells = W.c4_batched_cells(4, seed=11)
    for pos, q, lat in cells[:2]:
        pf, ff = oracle.fft_potential_force(pos, q, lat, 1e-10)
        pd, fd = oracle.direct_potential_force(pos, q, lat, 1e-12)
        assert rel_rms(pf, pd) < 1e-9
        assert rel_rms(ff, fd) < 1e-9


def test_madelung_constant(oracle):
    for d in (1.0, 2.5):
        pos, q, lat = W.perfect_rock_salt(4, d)
        pot = oracle.fft_potential_force(pos, q, lat, 1e-10, want_force=False)
        assert np.allclose(-pot * q * d, W.MADELUNG_NACL, rtol=0, atol=1e-9)


def test_force_is_minus_energy_gradient(oracle):
    rng = np.random.default_rng(3)
    pos, q, lat = W.random_cubic(16, 6.0, 5, "normal", 0.5)
    _, force = oracle.fft_potential_force(pos, q, lat, 1e-12)

    def energy(p):
        return 0.5 * np.dot(q, oracle.fft_potential_force(p, q, lat, 1e-12, want_force=False))

    h = 1e-5
    for i in rng.choice(len(q), 4, replace=False):
        for d in range(3):
            pp, pm = pos.copy(), pos.copy()
            pp[i, d] += h
            pm[i, d] -= h
            fd = -(energy(pp) - energy(pm)) / (2 * h)
            assert abs(fd - force[i, d]) < 1e-7 * max(1.0, np.abs(force).max())


def test_translation_invariance_and_zero_net_force(oracle):
    pos, q, lat = W.c1_small_cubic()
    p0, f0 = oracle.fft_potential_force(pos, q, lat, 1e-10)
    p1, f1 = oracle.fft_potential_force(pos + np.array([1.234, -0.5, 7.0]), q, lat, 1e-10)
    assert rel_max(p1, p0) < 1e-9 and rel_max(f1, f0) < 1e-9
    assert np.abs(f0.sum(axis=0)).max() < 1e-9 * np.abs(f0).max()


def test_stock_stress_is_strain_derivative(oracle):
    # invRStress returns sigma with TCoulomb%addStress doing stress -= sigma/2,
    # and DFTB+'s stress is -(1/V) dE/d(strain).  Hence sigma = (2/V) dE/deps
    # for the Ewald energy E = 1/2 sum q phi, checked with the direct engine.
    pos, q, lat = W.random_cubic(12, 5.0, 9, "normal", 0.5)
    lat = lat @ np.array([[1.0, 0.05, 0.0], [0.0, 1.0, 0.1], [0.02, 0.0, 1.0]])
    sigma, info = oracle.stock_stress(pos, q, lat.T, tol_ewald=1e-12)

    def energy(eps):
        F = np.eye(3) + eps
        p2 = pos @ F.T
        l2 = lat @ F.T
        return 0.5 * np.dot(q, oracle.direct_potential_force(p2, q, l2, 1e-13, want_force=False))

    V = abs(np.linalg.det(lat))
    h = 1e-5
    for a in range(3):
        for b in range(3):
            e = np.zeros((3, 3))
            e[a, b] = h
            dE = (energy(e) - energy(-e)) / (2 * h)
            assert abs(sigma[a, b] - 2.0 / V * dE) < 1e-7 * np.abs(sigma).max()
    assert info["n_g"] > 0 and info["alpha"] > 0


@pytest.mark.parametrize("case,code", [("charged", 3), ("tol", 4), ("volume", 5), ("coincident", 7),
                                        ("empty", 1)])
def test_error_statuses(oracle, case, code):
    pos, q, lat = W.c1_small_cubic()
    tol = 1e-10
    if case == "charged":
        q = q + 0.1
    elif case == "tol":
        tol = 1.5
    elif case == "volume":
        lat = np.zeros((3, 3))
    elif case == "coincident":
        pos = pos.copy()
        pos[5] = pos[3]
    elif case == "empty":
        pos, q = pos[:0], q[:0]
    with pytest.raises(oracle.OracleError) as ei:
        oracle.fft_potential_force(pos, q, lat, tol)
    assert ei.value.code == code


# ---- potentials and gradients at arbitrary points (stock Ewald) -------------

def _points_system(seed=3):
    pos, q, lat = W.c1_small_cubic()
    rng = np.random.default_rng(seed)
    targets = rng.uniform(0, 1, (6, 3)) @ lat
    return pos, q, lat, targets


def test_point_potential_at_the_atoms_is_the_shift(oracle):
    """getPotential at the charges themselves (neutral set) is the Ewald shift:
    the stock pair sum and the fast NFFT path agree to the tolerance."""
    pos, q, lat, _ = _points_system()
    p_stock = oracle.potential_at(pos, pos, q, lat.T, 1e-10)
    p_fast, _ = oracle.fft_potential_force(pos, q, lat, 1e-10)
    assert np.abs(p_stock - p_fast).max() / np.abs(p_fast).max() < 1e-9


@pytest.mark.parametrize("blur", [None, 0.8])
def test_point_gradient_is_the_derivative_of_the_potential(oracle, blur):
    pos, q, lat, tg = _points_system()
    b = None if blur is None else np.full(len(q), blur)
    g = oracle.potential_gradient_at(tg, pos, q, lat.T, 1e-10, blur=b)
    h = 1e-5
    fd = np.zeros_like(g)
    for d in range(3):
        e = np.zeros(3)
        e[d] = h
        fd[:, d] = (oracle.potential_at(tg + e, pos, q, lat.T, 1e-10, blur=b)
                    - oracle.potential_at(tg - e, pos, q, lat.T, 1e-10, blur=b)) / (2 * h)
    assert np.abs(g - fd).max() / np.abs(g).max() < 1e-8


def test_external_gradients_obey_newtons_third_law(oracle):
    pos, q, lat, tg = _points_system()
    qt = np.random.default_rng(4).normal(0, 0.3, len(tg))
    ga, ge = oracle.external_pot_grad(tg, pos, qt, q, lat.T, False, 1e-10)
    assert np.abs(ga.sum(0) + ge.sum(0)).max() < 1e-14 * np.abs(ga).max() * len(q)
    gh, _ = oracle.external_pot_grad(tg, pos, qt, q, lat.T, True, 1e-10)
    assert np.allclose(gh, oracle.potential_gradient_at(tg, pos, q, lat.T, 1e-10), rtol=0,
                       atol=1e-15)
    assert np.allclose(ga, qt[:, None] * gh, rtol=1e-13, atol=1e-16)


def test_softening_vanishes_far_away(oracle):
    pos, q, lat, tg = _points_system()
    p0 = oracle.potential_at(tg, pos, q, lat.T, 1e-10)
    p1 = oracle.potential_at(tg, pos, q, lat.T, 1e-10, eps_soften=1e-7)
    assert np.abs(p1 - p0).max() < 1e-10


def test_xlbomd_gradient_restatement(oracle):
    """addInvRPrimeXlbomdPeriodic: with qo = qi the shadow energy is the energy
    (gradient = -force of the fast path to the tolerance), and in general it is
    the gradient of E(qi + qo) - E(qo) - 2 E(qi)."""
    pos, q, lat = W.c1_small_cubic()
    g = oracle.xlbomd_gradients(pos, q, q, lat.T, 1e-10)
    _, f = oracle.fft_potential_force(pos, q, lat, 1e-10)
    assert np.abs(g + f).max() / np.abs(f).max() < 1e-8
    rng = np.random.default_rng(1)
    qo = q + rng.normal(0, 0.05, len(q))
    qo -= qo.mean()
    g = oracle.xlbomd_gradients(pos, q, qo, lat.T, 1e-10)
    f1 = oracle.fft_potential_force(pos, q + qo, lat, 1e-10)[1]
    f2 = oracle.fft_potential_force(pos, qo, lat, 1e-10)[1]
    f3 = oracle.fft_potential_force(pos, q, lat, 1e-10)[1]
    assert np.abs(g + (f1 - f2 - 2 * f3)).max() / np.abs(g).max() < 1e-8
