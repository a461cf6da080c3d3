"""The C ABI library without a GPU: it builds for sm_100a, loads, exports every
entry point include/ewald_b200.h declares, and its host-side parameter chain
matches the oracle exactly (integers bit for bit)."""

import ctypes as C
import os
import re

import numpy as np
import pytest

import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "ewald_b200.h")).read()
    return sorted(set(re.findall(r"\b(ewg_[a-z0-9_]+)\s*\(", text)))


def test_header_and_python_export_lists_agree(ewald_lib):
    assert declared_symbols() == sorted(ewald_lib.EXPORTED)


def test_library_exports_every_declared_symbol(ewald_lib):
    L = ewald_lib.lib()
    for name in declared_symbols():
        assert hasattr(L, name), name


def test_status_strings(ewald_lib):
    assert ewald_lib.status_string(0) == "ok"
    assert "neutral" in ewald_lib.status_string(3)
    assert "coincident" in ewald_lib.status_string(7)


CASES = [
    ("c1", W.c1_small_cubic, 1e-10, {}),
    ("c2", W.c2_random_4096, 1e-10, {}),
    ("c2_literal", W.c2_random_4096, 1e-10, {"r_cut_in": 10 * W.ANGSTROM_TO_BOHR, "nModes_in": 32}),
    ("c3", W.c3_water_32k, 1e-10, {}),
    ("c3_1e-6", W.c3_water_32k, 1e-6, {}),
    ("c5", W.c5_rock_salt_216k, 1e-10, {}),
    ("pair", W.reference_pair_fixture, 1e-9, {}),
    ("alpha_in", W.c1_small_cubic, 1e-10, {"alpha_in": 0.4}),
    ("kcut_window", W.c1_small_cubic, 1e-8, {"k_cut_in": 2.5, "windowCutoff_in": 7}),
]


@pytest.mark.parametrize("name,gen,tol,ov", CASES, ids=[c[0] for c in CASES])
def test_parameter_chain_matches_oracle(ewald_lib, oracle, name, gen, tol, ov):
    pos, q, lat = gen()
    got = ewald_lib.ewald_parameters(pos, q, len(q), lat, tol, **ov)
    okw = {{"alpha_in": "alpha", "r_cut_in": "r_cut", "k_cut_in": "k_cut", "nModes_in": "n_modes",
            "windowCutoff_in": "window_cutoff"}[k]: v for k, v in ov.items()}
    ref = oracle.fft_parameters(q, lat, tol, **okw)
    assert got["n_modes"] == ref["n_modes"]
    assert got["window_cutoff"] == ref["window_cutoff"]
    for k in ("alpha", "r_cut", "k_cut"):
        assert got[k] == pytest.approx(ref[k], rel=1e-15, abs=0.0)
    gb = ewald_lib.ewald_grid_memory(q, len(q), lat, tol, **ov)
    assert gb == pytest.approx(oracle.fft_grid_memory(q, lat, tol, **okw), rel=1e-14)


def test_host_side_errors(ewald_lib):
    pos, q, lat = W.c1_small_cubic()
    with pytest.raises(ewald_lib.EwaldError) as e:
        ewald_lib.ewald_parameters(pos, q + 0.1, len(q), lat, 1e-10)
    assert e.value.code == 3
    with pytest.raises(ewald_lib.EwaldError) as e:
        ewald_lib.ewald_parameters(pos, q, len(q), np.zeros((3, 3)), 1e-10)
    assert e.value.code == 5


def test_create_without_gpu_reports_no_device(ewald_lib):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    rc = ewald_lib.lib().ewg_create(C.byref(h), 0, 0)
    assert rc == 15  # EWG_ERR_NO_DEVICE, not a silent CPU path
