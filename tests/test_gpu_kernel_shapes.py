"""Kernel shapes (ewg_kernel_shape) and their autotuner (ewg_tune_kernels).

Every shape the tuner can pick is checked against the oracle at the plain
form's bar (1e-10 of the largest value).  The gather CTA shape and the FFT
lines per CTA change no arithmetic, so their results equal the default shape's
bitwise; the real-space box subdivision and the radix-4 FFT schedule reorder
sums, so their results move by rounding only.  The tuner's choice is cached per
bucket (precision form, force grids, atom octave, grid, window half-width) and
applied to every later evaluation in that bucket."""

import numpy as np
import pytest
from conftest import rel_max, rel_rms

import workloads as W

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10

# One field changed from the defaults at a time.
SHAPES = [
    ("box_div_1", {"box_div": 1}, False),
    ("box_div_3", {"box_div": 3}, False),
    ("gather_warps_2", {"gather_warps": 2}, True),
    ("gather_warps_8", {"gather_warps": 8}, True),
    ("fft_lines_4", {"fft_lines": 4}, True),
    ("fft_lines_2", {"fft_lines": 2}, True),
    ("fft_lines_1", {"fft_lines": 1}, True),
    ("fft_sched_radix4", {"fft_sched": 2}, False),
]


@pytest.fixture(scope="module")
def ctx(ewald_lib):
    c = ewald_lib.Context(0, ewald_lib.FP64)
    yield c
    c.close()


def triclinic(seed=21, n=300):
    rng = np.random.default_rng(seed)
    lat = W.triclinic_lattice(14.0, 17.0, 15.0, 78.0, 101.0, 95.0) * W.ANGSTROM_TO_BOHR
    pos = rng.uniform(0, 1, size=(n, 3)) @ lat
    q = rng.normal(0, 0.4, n)
    return pos, q - q.mean(), lat


# C1 is the image-sum regime (one reference-width box per axis, cutoff beyond half the cell).
SYSTEMS = [("c1", W.c1_small_cubic), ("c2", W.c2_random_4096), ("triclinic", triclinic)]


@pytest.mark.parametrize("sys_name,gen", SYSTEMS, ids=[s[0] for s in SYSTEMS])
@pytest.mark.parametrize("name,shape,bitwise", SHAPES, ids=[s[0] for s in SHAPES])
def test_every_shape_matches_oracle(ctx, oracle, sys_name, gen, name, shape, bitwise):
    pos, q, lat = gen()
    po, fo = oracle.fft_potential_force(pos, q, lat, 1e-10)
    ctx.set_kernel_shape({})  # defaults
    p0, f0 = ctx.potential_force(pos, q, lat, 1e-10)
    ctx.set_kernel_shape(shape)
    try:
        pg, fg = ctx.potential_force(pos, q, lat, 1e-10)
        pp = ctx.potential_force(pos, q, lat, 1e-10, want_force=False)
    finally:
        ctx.set_kernel_shape(None)
    assert rel_max(pg, po) < TOL_FP64, rel_max(pg, po)
    assert rel_max(fg, fo) < TOL_FP64, rel_max(fg, fo)
    assert rel_max(pp, po) < TOL_FP64
    if bitwise:
        assert np.array_equal(pg, p0) and np.array_equal(fg, f0)


def test_tune_kernels_caches_per_bucket(ewald_lib, ctx, oracle):
    pos, q, lat = W.c2_random_4096()
    ctx.potential_force(pos, q, lat, 1e-10)
    par = ctx.last_params()
    ov = {"alpha_in": par["alpha"], "r_cut_in": par["r_cut"], "k_cut_in": par["k_cut"],
          "windowCutoff_in": par["window_cutoff"]}
    shape, (ms_default, ms_tuned) = ctx.tune_kernels(pos, q, lat, 1e-10, **ov)
    assert ms_default > 0.0 and 0.0 < ms_tuned <= ms_default
    assert shape["box_div"] in (1, 2, 3) and shape["gather_warps"] in (2, 4, 8)
    assert shape["fft_lines"] in (0, 1, 2, 4, 8) and shape["fft_sched"] in (1, 2)
    # Another configuration of the same bucket (4096 <= n < 8192, same grid and
    # window through the same parameters): the cached shape, nothing evaluated.
    rng = np.random.default_rng(77)
    pos2 = rng.uniform(0, 1, size=(5000, 3)) @ lat
    q2 = rng.normal(0, 0.3, 5000)
    q2 -= q2.mean()
    launches = ctx.kernel_launches
    shape2, ms2 = ctx.tune_kernels(pos2, q2, lat, 1e-10, **ov)
    assert shape2 == shape and ms2 == (0.0, 0.0)
    assert ctx.kernel_launches == launches
    # Evaluations in the bucket run the tuned shape and keep the bar.
    pg, fg = ctx.potential_force(pos2, q2, lat, 1e-10, **ov)
    po, fo = oracle.fft_potential_force(pos2, q2, lat, 1e-10, alpha=par["alpha"],
                                        r_cut=par["r_cut"], k_cut=par["k_cut"],
                                        window_cutoff=par["window_cutoff"])
    assert rel_max(pg, po) < TOL_FP64
    assert rel_max(fg, fo) < TOL_FP64
    # A potential-only evaluation is another bucket: tuned anew.
    shape3, (ms3, _) = ctx.tune_kernels(pos, q, lat, 1e-10, want_force=False, **ov)
    assert ms3 > 0.0


@pytest.mark.parametrize("scheme", [0, 1], ids=["ik", "ad"])
def test_mixed_stencil_engines(ewald_lib, ctx, scheme):
    """The mixed form's spread and gathers on the FP64 tensor cores (default)
    and on the FP32 CUDA cores both stay within the mixed bar of the FP64 form."""
    pos, q, lat = W.water_box(1365, seed=3)
    p64, f64 = ctx.potential_force(pos, q, lat, 1e-10)
    cm = ewald_lib.Context(0, ewald_lib.MIXED)
    try:
        cm.set_force_scheme(scheme)
        out = {}
        for st in (1, 2):
            cm.set_kernel_shape({"stencil": st})
            out[st] = cm.potential_force(pos, q, lat, 1e-7)
            out[st, "pot"] = cm.potential_force(pos, q, lat, 1e-7, want_force=False)
    finally:
        cm.close()
    for st in (1, 2):
        pm, fm = out[st]
        assert rel_rms(fm, f64) < 1e-6 and rel_rms(pm, p64) < 1e-6
        assert rel_rms(out[st, "pot"], p64) < 1e-6
    # the tensor-core contraction is the more accurate of the two
    assert rel_rms(out[1][1], f64) <= 1.5 * rel_rms(out[2][1], f64)


def test_set_kernel_shape_rejects_bad_fields(ewald_lib, ctx):
    for bad in ({"box_div": 4}, {"fft_lines": 3}, {"fft_sched": 3}, {"gather_warps": 16},
                {"stencil": 3}):
        with pytest.raises(ewald_lib.EwaldError) as e:
            ctx.set_kernel_shape(bad)
        assert e.value.code == 2  # EWG_ERR_ARG
    ctx.set_kernel_shape(None)
