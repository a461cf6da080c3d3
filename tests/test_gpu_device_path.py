"""ewg_potential_force_device with overrides that fix alpha and k_cut: the
parameters then do not depend on the charges, the evaluation is queued behind
the device charge sums without a host wait, and neutrality is checked after the
call's synchronisation.  Results equal those of the host-array entry point with
the same overrides; a net charge still fails with EWG_ERR_NOT_NEUTRAL, and the
background convention (which needs the charge sum up front) still works."""

import numpy as np
import pytest
import torch

import workloads as W

pytestmark = pytest.mark.gpu

OV = {"alpha_in": 0.30, "r_cut_in": 11.0, "k_cut_in": 2.4, "windowCutoff_in": 8}


def _device(pos, q):
    x = torch.tensor(np.asarray(pos), dtype=torch.float64, device="cuda").contiguous()
    qq = torch.tensor(q, dtype=torch.float64, device="cuda").contiguous()
    pot = torch.empty(len(q), dtype=torch.float64, device="cuda")
    force = torch.empty((len(q), 3), dtype=torch.float64, device="cuda")
    return x, qq, pot, force


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_charge_independent_parameters_match_host_entry(ewald_lib, precision):
    pos, q, lat = W.c2_random_4096()
    ctx = ewald_lib.Context(0, getattr(ewald_lib, precision))
    try:
        hp, hf = ctx.potential_force(pos, q, lat, 1e-10, **OV)
        x, qq, pot, force = _device(pos, q)
        for _ in range(3):  # direct, record + replay, replay
            ctx.potential_force_device(x, qq, lat, 1e-10, pot, force, **OV)
            torch.cuda.synchronize()
            dp, df = pot.cpu().numpy(), force.cpu().numpy()
            assert np.max(np.abs(dp - hp)) <= 1e-12 * np.max(np.abs(hp))
            assert np.max(np.abs(df - hf)) <= 1e-12 * np.max(np.abs(hf))
        assert ctx.last_params()["alpha"] == OV["alpha_in"]
    finally:
        ctx.close()


def test_net_charge_still_refused(ewald_lib):
    pos, q, lat = W.c2_random_4096()
    q = np.asarray(q).copy()
    q[0] += 0.5
    ctx = ewald_lib.Context(0, ewald_lib.FP64)
    try:
        x, qq, pot, force = _device(pos, q)
        with pytest.raises(ewald_lib.EwaldError) as ei:
            ctx.potential_force_device(x, qq, lat, 1e-10, pot, force, **OV)
        assert ei.value.code == 3  # EWG_ERR_NOT_NEUTRAL
        # the context stays usable
        q[0] -= 0.5
        x, qq, pot, force = _device(pos, q)
        ctx.potential_force_device(x, qq, lat, 1e-10, pot, force, **OV)
        torch.cuda.synchronize()
        assert np.all(np.isfinite(pot.cpu().numpy()))
    finally:
        ctx.close()


def test_background_with_fixed_parameters(ewald_lib):
    pos, q, lat = W.c2_random_4096()
    q = np.asarray(q).copy()
    q[0] += 0.5
    ctx = ewald_lib.Context(0, ewald_lib.FP64)
    try:
        ctx.set_background(True)
        hp, hf = ctx.potential_force(pos, q, lat, 1e-10, **OV)
        x, qq, pot, force = _device(pos, q)
        ctx.potential_force_device(x, qq, lat, 1e-10, pot, force, **OV)
        torch.cuda.synchronize()
        assert np.max(np.abs(pot.cpu().numpy() - hp)) <= 1e-12 * np.max(np.abs(hp))
        assert np.max(np.abs(force.cpu().numpy() - hf)) <= 1e-12 * np.max(np.abs(hf))
    finally:
        ctx.close()


def test_host_entry_with_fixed_parameters(ewald_lib, oracle):
    """The host-array entry point with alpha and k_cut fixed checks the charges
    while the evaluation runs: results match the oracle at those parameters,
    and a net charge still fails with EWG_ERR_NOT_NEUTRAL."""
    pos, q, lat = W.c1_small_cubic()
    ov = {"alpha_in": 0.30, "r_cut_in": 11.0, "k_cut_in": 2.4, "windowCutoff_in": 10}
    ctx = ewald_lib.Context(0, ewald_lib.FP64)
    try:
        for _ in range(3):  # direct, record + replay, replay
            pot, force = ctx.potential_force(pos, q, lat, 1e-10, **ov)
        po, fo = oracle.fft_potential_force(pos, q, lat, 1e-10, alpha=0.30, r_cut=11.0, k_cut=2.4,
                                            window_cutoff=10)
        assert np.max(np.abs(pot - po)) <= 1e-10 * np.max(np.abs(po))
        assert np.max(np.abs(force - fo)) <= 1e-10 * np.max(np.abs(fo))
        bad = np.asarray(q).copy()
        bad[0] += 0.5
        with pytest.raises(ewald_lib.EwaldError) as ei:
            ctx.potential_force(pos, bad, lat, 1e-10, **ov)
        assert ei.value.code == 3  # EWG_ERR_NOT_NEUTRAL
    finally:
        ctx.close()
