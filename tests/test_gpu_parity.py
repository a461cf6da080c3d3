"""GPU parity: the CUDA library (through its C ABI) against the CPU oracle on the
same seeded inputs.  Plain FP64 form: max |difference| / max |reference| below
1e-10 for potential, force and stress (the reference's stated bar).  Mixed
form: RMS force error below 1e-6 relative to the FP64 result."""

import numpy as np
import pytest
from conftest import rel_max, rel_rms

import workloads as W

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10   # plain form vs oracle, relative to max |reference|
TOL_MIXED_RMS = 1e-6


@pytest.fixture(scope="module")
def ctx(ewald_lib):
    c = ewald_lib.Context(0, ewald_lib.FP64)
    yield c
    c.close()


@pytest.fixture(scope="module")
def ctx_mixed(ewald_lib):
    c = ewald_lib.Context(0, ewald_lib.MIXED)
    yield c
    c.close()


def small_triclinic(seed=21, n=300):
    rng = np.random.default_rng(seed)
    lat = W.triclinic_lattice(14.0, 17.0, 15.0, 78.0, 101.0, 95.0) * W.ANGSTROM_TO_BOHR
    pos = rng.uniform(0, 1, size=(n, 3)) @ lat + rng.normal(0, 30, size=3)
    q = rng.normal(0, 0.4, n)
    return pos, q - q.mean(), lat


CASES = [
    ("c1_image_sum", W.c1_small_cubic, 1e-10, {}),
    ("pair_fixture", W.reference_pair_fixture, 1e-9, {}),
    ("triclinic", small_triclinic, 1e-10, {}),
    ("c2_chain", W.c2_random_4096, 1e-10, {}),
    ("c2_literal", W.c2_random_4096, 1e-10, {"r_cut": 10 * W.ANGSTROM_TO_BOHR, "n_modes": 32}),
    ("c2_tol1e-6", W.c2_random_4096, 1e-6, {}),
    ("odd_modes", small_triclinic, 1e-8, {"n_modes": 15, "window_cutoff": 6}),
    ("small_grid_wraps", W.c1_small_cubic, 1e-8, {"n_modes": 6}),
]

OV_NAMES = {"alpha": "alpha_in", "r_cut": "r_cut_in", "k_cut": "k_cut_in", "n_modes": "nModes_in",
            "window_cutoff": "windowCutoff_in"}


@pytest.mark.parametrize("name,gen,tol,ov", CASES, ids=[c[0] for c in CASES])
def test_fp64_matches_oracle(ctx, oracle, name, gen, tol, ov):
    pos, q, lat = gen()
    pg, fg = ctx.potential_force(pos, q, lat, tol, **{OV_NAMES[k]: v for k, v in ov.items()})
    po, fo = oracle.fft_potential_force(pos, q, lat, tol, **ov)
    assert rel_max(pg, po) < TOL_FP64, rel_max(pg, po)
    assert rel_max(fg, fo) < TOL_FP64, rel_max(fg, fo)


def elongated_cell(dims_angstrom, n=64, seed=5):
    lat = np.diag(dims_angstrom) * W.ANGSTROM_TO_BOHR
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, 1, size=(n, 3)) @ lat
    q = rng.normal(0, 0.5, n)
    return pos, q - q.mean(), lat


# Cells with one long axis and a 20 Angstrom cutoff give FFT lines of 1680-3360
# points: in FP64 their passes hold 2 or 1 lines per CTA instead of 4 or 8.
LONG_AXIS_CASES = [
    ("x3360", (3000.0, 8.0, 8.0)),   # x passes, one line per CTA
    ("x2000", (1800.0, 8.0, 8.0)),   # x passes, two lines
    ("y2000", (8.0, 1800.0, 8.0)),   # y passes, two lines
    ("z2688", (8.0, 8.0, 2400.0)),   # fused z pass, one line
    ("z1680", (8.0, 8.0, 1500.0)),   # fused z pass, two lines
]


@pytest.mark.parametrize("dims", [c[1] for c in LONG_AXIS_CASES], ids=[c[0] for c in LONG_AXIS_CASES])
def test_long_axes_match_oracle(ctx, ctx_mixed, oracle, dims):
    pos, q, lat = elongated_cell(dims)
    r_cut = 20.0 * W.ANGSTROM_TO_BOHR
    po, fo = oracle.fft_potential_force(pos, q, lat, 1e-10, r_cut=r_cut)
    pg, fg = ctx.potential_force(pos, q, lat, 1e-10, r_cut_in=r_cut)
    assert rel_max(pg, po) < TOL_FP64, rel_max(pg, po)
    assert rel_max(fg, fo) < TOL_FP64, rel_max(fg, fo)
    pm, fm = ctx_mixed.potential_force(pos, q, lat, 1e-10, r_cut_in=r_cut)
    assert rel_rms(fm, fo) < TOL_MIXED_RMS
    assert rel_rms(pm, po) < TOL_MIXED_RMS


def test_potential_only_matches_oracle(ctx, oracle):
    pos, q, lat = W.c2_random_4096()
    pg = ctx.potential_force(pos, q, lat, 1e-10, want_force=False)
    po = oracle.fft_potential_force(pos, q, lat, 1e-10, want_force=False)
    assert rel_max(pg, po) < TOL_FP64


def test_reference_shaped_call(ewald_lib, oracle):
    pos, q, lat = W.c1_small_cubic()
    n = len(q)
    pot = np.zeros(n)
    force = np.zeros((3, n))
    ewald_lib.ewald_potential_force(pos, q, n, lat, 1e-10, pot, force)
    po, fo = oracle.fft_potential_force(pos, q, lat, 1e-10)
    assert rel_max(pot, po) < TOL_FP64
    assert rel_max(force.T, fo) < TOL_FP64


def test_bitwise_deterministic(ctx):
    pos, q, lat = W.c2_random_4096()
    a = ctx.potential_force(pos, q, lat, 1e-10)
    b = ctx.potential_force(pos, q, lat, 1e-10)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_direct_engine_matches_oracle(ctx, oracle):
    for gen in (W.c1_small_cubic, lambda: small_triclinic(5, 120)):
        pos, q, lat = gen()
        pg, fg = ctx.direct_potential_force(pos, q, lat, 1e-12)
        po, fo = oracle.direct_potential_force(pos, q, lat, 1e-12)
        assert rel_max(pg, po) < TOL_FP64
        assert rel_max(fg, fo) < TOL_FP64


def test_stock_stress_matches_oracle(ctx, oracle):
    for gen, tol in ((W.c1_small_cubic, 1e-10), (W.reference_pair_fixture, 1e-9),
                     (lambda: small_triclinic(8, 200), 1e-9)):
        pos, q, lat = gen()
        ctx.set_lattice(lat.T)
        ctx.set_coords(pos)
        ctx.set_charges(q)
        sg = ctx.stress(tol)
        so, info = oracle.stock_stress(pos, q, lat.T, tol)
        assert rel_max(sg, so) < TOL_FP64, (rel_max(sg, so), sg, so)
        setup = ctx.last_stress_setup()
        assert setup["n_g"] == info["n_g"]
        assert setup["alpha"] == pytest.approx(info["alpha"], rel=1e-15)


def test_tcoulomb_scc_sequence(ewald_lib, oracle):
    pos, q, lat = W.c2_random_4096()
    n = len(q)
    tc = ewald_lib.TCoulomb(n, tolEwald=1e-10)
    tc.updateLatVecs(lat.T)
    tc.updateCoords(pos.T)
    rng = np.random.default_rng(0)
    for it in range(3):  # SCC iterations: only the charges move
        dq = q * (1.0 + 0.1 * it) + rng.normal(0, 0.01, n)
        dq -= dq.mean()
        tc.updateCharges(dq)
        shift = tc.updateShifts()
        po = oracle.fft_potential_force(pos, dq, lat, 1e-10, want_force=False)
        assert rel_max(shift, po) < TOL_FP64
        e = np.zeros(n)
        tc.addEnergy(e)
        assert np.allclose(e, 0.5 * shift * dq)
    grad = np.zeros((3, n))
    tc.addGradients(grad)
    _, fo = oracle.fft_potential_force(pos, dq, lat, 1e-10)
    assert rel_max(-grad.T, fo) < TOL_FP64
    stress = np.zeros((3, 3))
    tc.addStress(stress)
    so, _ = oracle.stock_stress(pos, dq, lat.T, 1e-10)
    assert rel_max(stress, -0.5 * so) < TOL_FP64


def test_batched_cells_match_oracle(ctx, oracle):
    cells = W.c4_batched_cells(6, seed=4)
    pots, forces = ctx.batch_potential_force(cells, 1e-10)
    for (pos, q, lat), pg, fg in zip(cells, pots, forces):
        po, fo = oracle.fft_potential_force(pos, q, lat, 1e-10)
        assert rel_max(pg, po) < TOL_FP64
        assert rel_max(fg, fo) < TOL_FP64


def test_device_pointer_entry(ctx, oracle):
    torch = pytest.importorskip("torch")
    pos, q, lat = W.c1_small_cubic()
    x = torch.tensor(pos, dtype=torch.float64, device="cuda").contiguous()
    qq = torch.tensor(q, dtype=torch.float64, device="cuda")
    pot = torch.empty(len(q), dtype=torch.float64, device="cuda")
    force = torch.empty((len(q), 3), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.potential_force_device(x, qq, lat, 1e-10, pot, force)
    po, fo = oracle.fft_potential_force(pos, q, lat, 1e-10)
    assert rel_max(pot.cpu().numpy(), po) < TOL_FP64
    assert rel_max(force.cpu().numpy(), fo) < TOL_FP64


def test_mixed_form_error_vs_fp64(ctx, ctx_mixed):
    pos, q, lat = W.c2_random_4096()
    p64, f64 = ctx.potential_force(pos, q, lat, 1e-10)
    p32, f32 = ctx_mixed.potential_force(pos, q, lat, 1e-10)
    assert rel_rms(f32, f64) < TOL_MIXED_RMS
    assert rel_rms(p32, p64) < TOL_MIXED_RMS


@pytest.mark.parametrize("case,code", [("charged", 3), ("tol", 4), ("volume", 5), ("coincident", 7),
                                        ("empty", 1)])
def test_error_statuses(ctx, ewald_lib, case, code):
    pos, q, lat = W.c1_small_cubic()
    tol = 1e-10
    if case == "charged":
        q = q + 0.1
    elif case == "tol":
        tol = 0.0
    elif case == "volume":
        lat = np.zeros((3, 3))
    elif case == "coincident":
        pos = pos.copy()
        pos[7] = pos[2]
    elif case == "empty":
        pos, q = pos[:0], q[:0]
    with pytest.raises(ewald_lib.EwaldError) as ei:
        ctx.potential_force(pos, q, lat, tol)
    assert ei.value.code == code
    # The context stays usable after an error.
    pos, q, lat = W.c1_small_cubic()
    ctx.potential_force(pos, q, lat, 1e-10)


def test_native_kernels_launched(ctx):
    before = ctx.kernel_launches
    pos, q, lat = W.c1_small_cubic()
    ctx.potential_force(pos, q, lat, 1e-10)
    assert ctx.kernel_launches - before >= 10
