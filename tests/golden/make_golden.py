"""Regenerate tests/golden/oracle_fixtures.npz (TEST INFRASTRUCTURE).

The fixtures are outputs of the CPU oracle (oracle/, a restatement of the
reference's fast Ewald library and stock stress) on seeded inputs, so that the
oracle itself and the CUDA library can be checked against frozen values.  The
reference has no golden vectors of its own for this path (parity unpinned); the
oracle is pinned separately by tests/test_oracle.py.

Run from the repository root:  python tests/golden/make_golden.py
"""

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "dftb_fast-ewald_3d_b200"))

import oracle  # noqa: E402
import workloads as W  # noqa: E402


def triclinic_100():
    rng = np.random.default_rng(77)
    lat = W.triclinic_lattice(11.0, 13.0, 12.0, 80.0, 97.0, 104.0) * W.ANGSTROM_TO_BOHR
    pos = rng.uniform(0, 1, size=(100, 3)) @ lat
    q = rng.normal(0, 0.4, 100)
    return pos, q - q.mean(), lat


CASES = {
    "c1": (W.c1_small_cubic, 1e-10),
    "pair": (W.reference_pair_fixture, 1e-9),
    "tric100": (triclinic_100, 1e-10),
}


def main():
    oracle.build()
    out = {}
    for name, (gen, tol) in CASES.items():
        pos, q, lat = gen()
        pot, force = oracle.fft_potential_force(pos, q, lat, tol)
        sigma, info = oracle.stock_stress(pos, q, lat.T, tol)
        p = oracle.fft_parameters(q, lat, tol)
        out[f"{name}_pos"] = pos
        out[f"{name}_q"] = q
        out[f"{name}_lat"] = lat
        out[f"{name}_tol"] = np.array(tol)
        out[f"{name}_pot"] = pot
        out[f"{name}_force"] = force
        out[f"{name}_stress"] = sigma
        out[f"{name}_modes"] = np.array(p["n_modes"])
        out[f"{name}_window"] = np.array(p["window_cutoff"])
        out[f"{name}_alpha"] = np.array(p["alpha"])
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_fixtures.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    main()
