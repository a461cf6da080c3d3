"""Frozen oracle outputs (tests/golden/make_golden.py): the oracle must keep
reproducing them, and the CUDA library must match them to 1e-10."""

import os

import numpy as np
import pytest
from conftest import rel_max

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = np.load(os.path.join(HERE, "golden", "oracle_fixtures.npz"))
NAMES = ["c1", "pair", "tric100"]


def case(name):
    return (FIX[f"{name}_pos"], FIX[f"{name}_q"], FIX[f"{name}_lat"], float(FIX[f"{name}_tol"]))


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_fixture(oracle, name):
    pos, q, lat, tol = case(name)
    pot, force = oracle.fft_potential_force(pos, q, lat, tol)
    assert rel_max(pot, FIX[f"{name}_pot"]) < 1e-13
    assert rel_max(force, FIX[f"{name}_force"]) < 1e-13
    sigma, _ = oracle.stock_stress(pos, q, lat.T, tol)
    assert rel_max(sigma, FIX[f"{name}_stress"]) < 1e-12
    p = oracle.fft_parameters(q, lat, tol)
    assert tuple(FIX[f"{name}_modes"]) == p["n_modes"]
    assert int(FIX[f"{name}_window"]) == p["window_cutoff"]


@pytest.mark.parametrize("name", NAMES)
def test_library_parameters_match_fixture(ewald_lib, name):
    pos, q, lat, tol = case(name)
    p = ewald_lib.ewald_parameters(pos, q, len(q), lat, tol)
    assert tuple(FIX[f"{name}_modes"]) == p["n_modes"]
    assert int(FIX[f"{name}_window"]) == p["window_cutoff"]
    assert p["alpha"] == pytest.approx(float(FIX[f"{name}_alpha"]), rel=1e-15)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_matches_fixture(ewald_lib, name):
    pos, q, lat, tol = case(name)
    ctx = ewald_lib.Context(0, ewald_lib.FP64)
    try:
        pot, force = ctx.potential_force(pos, q, lat, tol)
        ctx.set_lattice(lat.T)
        ctx.set_coords(pos)
        ctx.set_charges(q)
        sigma = ctx.stress(tol)
    finally:
        ctx.close()
    assert rel_max(pot, FIX[f"{name}_pot"]) < 1e-10
    assert rel_max(force, FIX[f"{name}_force"]) < 1e-10
    assert rel_max(sigma, FIX[f"{name}_stress"]) < 1e-10
