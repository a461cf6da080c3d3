"""The C ABI library without a GPU: it builds for sm_100a, loads, exports every
entry point include/ewald_b200.h declares, and its host-side parameter chain
matches the oracle exactly (integers bit for bit)."""

import ctypes as C
import os
import re
import shutil
import subprocess

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


def _cc():
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    return cc


def test_header_is_c99_and_the_c_driver_links(tmp_path, ewald_lib):
    """The plain C caller (tests/c_driver) builds against the header alone and
    links every entry point it uses; it is run by the GPU tests."""
    ewald_lib.lib()
    libdir = os.path.join(ROOT, "dftb_fast-ewald_3d_b200")
    subprocess.run([_cc(), "-std=c99", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_driver", "tcoulomb_sequence.c"), "-L", libdir,
                    "-lewald_b200", f"-Wl,-rpath,{libdir}", "-o", str(tmp_path / "driver")],
                   check=True)


def test_struct_layouts_match_the_python_mirror(tmp_path, ewald_lib):
    """Sizes and member offsets of the header's structs as a C compiler lays
    them out, against the ctypes structures of the Python mirror."""
    members = {"ewg_overrides": ("Overrides", ["has_alpha", "has_window_cutoff", "alpha", "r_cut",
                                               "k_cut", "n_modes", "window_cutoff"]),
               "ewg_params": ("Params", ["alpha", "k_cut", "window_cutoff", "n_modes"]),
               "ewg_kernel_shape": ("KernelShape", ["box_div", "fft_lines", "fft_sched",
                                                    "gather_warps", "stencil"])}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "ewald_b200.h"', 'int main(void) {']
    for cname, (_, fields) in members.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in fields:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = str(tmp_path / "layout")
    subprocess.run([_cc(), "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", exe], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, (pyname, fields) in members.items():
        py = getattr(ewald_lib, pyname)
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f in fields:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


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
