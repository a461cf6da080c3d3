"""Replay of evaluation launch sequences as CUDA graphs (ewg_set_graphs): the
replayed evaluations give bitwise the results of direct launches through the
same entry point, follow new input values behind the same device pointers,
count their kernels, and survive buffer reallocation by a larger system in
between."""

import numpy as np
import pytest
import torch

import workloads as W

pytestmark = pytest.mark.gpu


def _device_inputs(pos, q):
    x = torch.tensor(np.asarray(pos), dtype=torch.float64, device="cuda").contiguous()
    qq = torch.tensor(q, dtype=torch.float64, device="cuda").contiguous()
    pot = torch.empty(len(q), dtype=torch.float64, device="cuda")
    force = torch.empty((len(q), 3), dtype=torch.float64, device="cuda")
    return x, qq, pot, force


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_replay_matches_direct_launches(ewald_lib, precision):
    prec = getattr(ewald_lib, precision)
    pos, q, lat = W.c2_random_4096()
    graphs = ewald_lib.Context(0, prec)
    direct = ewald_lib.Context(0, prec)
    direct.set_graphs(False)
    try:
        x, qq, pot, force = _device_inputs(pos, q)
        _, _, rpot, rforce = _device_inputs(pos, q)
        direct.potential_force_device(x, qq, lat, 1e-10, rpot, rforce)
        torch.cuda.synchronize()
        ref_pot, ref_force = rpot.cpu().numpy(), rforce.cpu().numpy()
        counts = []
        for _ in range(4):  # direct, record + replay, replay, replay
            before = graphs.kernel_launches
            graphs.potential_force_device(x, qq, lat, 1e-10, pot, force)
            torch.cuda.synchronize()
            counts.append(graphs.kernel_launches - before)
            assert np.array_equal(pot.cpu().numpy(), ref_pot)
            assert np.array_equal(force.cpu().numpy(), ref_force)
        assert len(set(counts)) == 1 and counts[0] > 10
        # new positions behind the same pointers: the replay reads them
        pos2 = np.asarray(pos) + np.array([0.3, -0.2, 0.1])
        x.copy_(torch.tensor(pos2, dtype=torch.float64, device="cuda"))
        graphs.potential_force_device(x, qq, lat, 1e-10, pot, force)
        direct.potential_force_device(x, qq, lat, 1e-10, rpot, rforce)
        torch.cuda.synchronize()
        assert torch.equal(pot, rpot) and torch.equal(force, rforce)
        assert not np.array_equal(pot.cpu().numpy(), ref_pot)  # the new positions took effect
    finally:
        graphs.close()
        direct.close()


def test_replay_after_reallocation(ewald_lib):
    small = W.c2_random_4096()
    big = W.water_box(2730, seed=3)
    ctx = ewald_lib.Context(0, ewald_lib.FP64)
    ref = ewald_lib.Context(0, ewald_lib.FP64)
    ref.set_graphs(False)
    try:
        for pos, q, lat in (small, small, small, big, big, big, small, small, small):
            pg, fg = ctx.potential_force(pos, q, lat, 1e-10)
            pr, fr = ref.potential_force(pos, q, lat, 1e-10)
            assert np.array_equal(pg, pr) and np.array_equal(fg, fr)
    finally:
        ctx.close()
        ref.close()
