"""Seeded synthetic inputs with the shapes of the five benchmark configurations.

No public dataset exists for this path; these generators stand in for it.  Sizes
are given in Angstrom, as the configurations are specified, and converted to
Bohr (atomic units) before any call, exactly as DFTB+ passes atomic units to the
Coulomb operator (src/dftbp/dftb/coulomb.F90:336-357).

Every generator returns ``positions`` (N, 3) in Bohr with one atom per row,
``charges`` (N,) summing to zero, and ``lat_rows`` (3, 3) in Bohr with one
lattice vector per row (the convention of ewald_potential_force,
src/dftbp/extlibs/fftewald/fft/ewald_fft_3d.f90:36-50).
"""

from __future__ import annotations

import math

import numpy as np

ANGSTROM_TO_BOHR = 1.8897261254578281


def _neutral(q):
    q = np.asarray(q, dtype=np.float64)
    return q - q.mean()


def random_cubic(n: int, box_angstrom: float, seed: int, charge: str = "uniform", sigma: float = 0.3):
    rng = np.random.default_rng(seed)
    L = box_angstrom * ANGSTROM_TO_BOHR
    pos = rng.uniform(0.0, L, size=(n, 3))
    if charge == "uniform":
        q = rng.uniform(-0.5, 0.5, size=n)
    else:
        q = rng.normal(0.0, sigma, size=n)
    return pos, _neutral(q), np.eye(3) * L


def c1_small_cubic():
    """64 charges, L = 12 Angstrom, q ~ U[-0.5, 0.5] minus the mean, seed 1."""
    return random_cubic(64, 12.0, 1, "uniform")


def c2_random_4096():
    """4096 charges, L = 35 Angstrom, q ~ N(0, 0.3) minus the mean, seed 2."""
    return random_cubic(4096, 35.0, 2, "normal", 0.3)


def _random_rotations(rng, n):
    quat = rng.normal(size=(n, 4))
    quat /= np.linalg.norm(quat, axis=1, keepdims=True)
    w, x, y, z = quat.T
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def water_box(n_molecules: int = 10923, density_g_cm3: float = 1.0, seed: int = 3):
    """Rigid 3-site waters (O -0.82, H +0.41, O-H 0.96 A, HOH 104.5 deg).

    Molecules sit on a jittered simple-cubic lattice (O-O >= 2.5 A is guaranteed
    by keeping each jitter component below (spacing - 2.5 A)/2) with uniformly random
    orientations; the cubic cell is sized for the requested mass density."""
    rng = np.random.default_rng(seed)
    mass = 18.015 / 6.02214076e23  # g per molecule
    volume_cm3 = n_molecules * mass / density_g_cm3
    L_ang = (volume_cm3 * 1e24) ** (1.0 / 3.0)
    per_axis = math.ceil(n_molecules ** (1.0 / 3.0))
    spacing = L_ang / per_axis
    sites = np.stack(np.meshgrid(*(np.arange(per_axis),) * 3, indexing="ij"), -1).reshape(-1, 3)
    chosen = sites[np.sort(rng.choice(sites.shape[0], n_molecules, replace=False))]
    jitter = rng.uniform(-1.0, 1.0, size=(n_molecules, 3)) * (0.5 * (spacing - 2.5))
    oxy = (chosen + 0.5) * spacing + jitter
    half = math.radians(104.5) / 2.0
    local_h = 0.96 * np.array([[math.sin(half), math.cos(half), 0.0],
                               [-math.sin(half), math.cos(half), 0.0]])
    R = _random_rotations(rng, n_molecules)
    h = oxy[:, None, :] + np.einsum("nij,hj->nhi", R, local_h)
    pos = np.empty((n_molecules, 3, 3))
    pos[:, 0] = oxy
    pos[:, 1:] = h
    pos = pos.reshape(-1, 3) * ANGSTROM_TO_BOHR
    q = np.tile(np.array([-0.82, 0.41, 0.41]), n_molecules)
    return pos, q.astype(np.float64), np.eye(3) * (L_ang * ANGSTROM_TO_BOHR)


def c3_water_32k():
    """10,923 waters = 32,769 atoms at 1.0 g/cm^3 (L = 68.91 Angstrom), seed 3."""
    return water_box(10923, 1.0, 3)


def triclinic_lattice(a, b, c, alpha_deg, beta_deg, gamma_deg):
    """Lattice vectors (rows) from cell lengths and angles, or None if invalid."""
    al, be, ga = (math.radians(x) for x in (alpha_deg, beta_deg, gamma_deg))
    ax = np.array([a, 0.0, 0.0])
    bx = np.array([b * math.cos(ga), b * math.sin(ga), 0.0])
    cx = c * math.cos(be)
    cy = c * (math.cos(al) - math.cos(be) * math.cos(ga)) / math.sin(ga)
    cz2 = c * c - cx * cx - cy * cy
    if cz2 <= 1e-6 * c * c:
        return None
    return np.array([ax, bx, [cx, cy, math.sqrt(cz2)]])


def c4_batched_cells(n_cells: int = 256, seed: int = 4):
    """Independent triclinic cells: N_c log-uniform in [50, 2000], lengths
    U[10, 30] A, angles U[70, 110] deg (invalid metrics rejected), q ~ N(0, 0.4)
    zero-sum per cell.  Returns a list of (positions, charges, lat_rows)."""
    rng = np.random.default_rng(seed)
    cells = []
    while len(cells) < n_cells:
        n = int(round(math.exp(rng.uniform(math.log(50), math.log(2000)))))
        lens = rng.uniform(10.0, 30.0, size=3)
        angs = rng.uniform(70.0, 110.0, size=3)
        lat = triclinic_lattice(*lens, *angs)
        if lat is None:
            continue
        lat = lat * ANGSTROM_TO_BOHR
        frac = rng.uniform(0.0, 1.0, size=(n, 3))
        pos = frac @ lat
        q = _neutral(rng.normal(0.0, 0.4, size=n))
        cells.append((pos, q, lat))
    return cells


def rock_salt(sites_per_axis: int = 60, nn_spacing_angstrom: float = 2.82, seed: int = 5,
              charge_jitter: float = 0.05, position_jitter_angstrom: float = 0.05):
    """Rock-salt supercell of sites_per_axis^3 sites, charges +-0.8 with
    N(0, charge_jitter) jitter renormalised to zero net charge, positions jittered
    by N(0, position_jitter) Angstrom."""
    rng = np.random.default_rng(seed)
    idx = np.stack(np.meshgrid(*(np.arange(sites_per_axis),) * 3, indexing="ij"), -1).reshape(-1, 3)
    sign = np.where(idx.sum(axis=1) % 2 == 0, 1.0, -1.0)
    pos = idx * nn_spacing_angstrom + rng.normal(0.0, position_jitter_angstrom, size=idx.shape)
    q = _neutral(0.8 * sign + rng.normal(0.0, charge_jitter, size=sign.shape))
    L = sites_per_axis * nn_spacing_angstrom * ANGSTROM_TO_BOHR
    return pos * ANGSTROM_TO_BOHR, q, np.eye(3) * L


def c5_rock_salt_216k():
    """60^3 rock-salt sites, a = 2.82 Angstrom, seed 5."""
    return rock_salt(60, 2.82, 5)


def c5_charge_update(base_charges, k: int):
    """k-th SCC-style charge update of the rock-salt workload (seed 5 + k),
    keeping the sign pattern and neutrality."""
    rng = np.random.default_rng(5 + k)
    sign = np.sign(base_charges)
    return _neutral(0.8 * sign + rng.normal(0.0, 0.05, size=sign.shape))


def charge_update(base_charges, k: int, seed: int, scale: float = 0.05):
    """k-th SCC-style charge update of a workload (seed + k): each charge
    moves by N(0, scale) relative to its own size, neutrality kept."""
    rng = np.random.default_rng(seed + k)
    q = np.asarray(base_charges, dtype=np.float64)
    return _neutral(q * (1.0 + rng.normal(0.0, scale, size=q.shape)))


def reference_pair_fixture():
    """The 2-atom periodic fixture of the reference's unit test
    (test/src/dftbp/unit/dftb/coulomb.F90:104-195): lattice diag(2,1,1) Bohr,
    charges +1/-1, x separation 1.1 Bohr, tolerance 1e-9."""
    pos = np.array([[0.0, 0.0, 0.0], [1.1, 0.0, 0.0]])
    return pos, np.array([1.0, -1.0]), np.diag([2.0, 1.0, 1.0])


def perfect_rock_salt(sites_per_axis: int = 4, spacing_bohr: float = 1.0):
    """Unjittered rock-salt with charges +-1: the site potential is
    -M * q / d with the Madelung constant M = 1.747564594633182."""
    idx = np.stack(np.meshgrid(*(np.arange(sites_per_axis),) * 3, indexing="ij"), -1).reshape(-1, 3)
    q = np.where(idx.sum(axis=1) % 2 == 0, 1.0, -1.0)
    return idx * spacing_bohr, q, np.eye(3) * sites_per_axis * spacing_bohr


MADELUNG_NACL = 1.747564594633182
