"""Host logic of the multi-rank batched form, on CPU: the LPT partition and a
world_size-2 gloo run whose gathered results equal the single-process ones
(the per-rank evaluator is the oracle; no GPU involved)."""

import os
import socket

import numpy as np
import pytest

import sharding
import workloads as W


def test_partition_is_a_balanced_cover():
    rng = np.random.default_rng(0)
    costs = list(rng.uniform(1, 100, size=37))
    for ws in (1, 2, 3, 8):
        shards = sharding.partition(costs, ws)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(costs) + 1e-9
    assert sharding.partition([5.0, 5.0, 5.0], 2) == [[0, 2], [1]]


def _params(pos, q, lat, tol):
    import oracle

    return oracle.fft_parameters(q, lat, tol)


def _evaluate(cells, tol):
    import oracle

    pots, forces = [], []
    for pos, q, lat in cells:
        p, f = oracle.fft_potential_force(pos, q, lat, tol)
        pots.append(p)
        forces.append(f)
    return pots, forces


def _worker(rank, world, port, cells, tol, out_path):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    for p in (os.path.join(root, "dftb_fast-ewald_3d_b200"), os.path.join(root, "oracle"), here):
        sys.path.insert(0, p)
    import torch.distributed as dist

    import sharding as sh

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pots, forces = sh.run_sharded(cells, tol, _evaluate, _params, rank, world)
        np.savez(out_path + f".{rank}.npz", *pots, *forces)
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_rank_gloo_matches_single_process(tmp_path, oracle):
    import torch.multiprocessing as mp

    cells = W.c4_batched_cells(5, seed=13)
    cells = [(p[:120], q[:120] - q[:120].mean(), l) for p, q, l in cells]
    tol = 1e-8
    out = str(tmp_path / "res")
    mp.start_processes(_worker, args=(2, _free_port(), cells, tol, out), nprocs=2, join=True,
                       start_method="spawn")
    ref_p, ref_f = _evaluate(cells, tol)
    for rank in range(2):
        d = np.load(out + f".{rank}.npz")
        arrs = [d[f"arr_{i}"] for i in range(len(d.files))]
        pots, forces = arrs[: len(cells)], arrs[len(cells):]
        # The oracle's OpenMP spread uses atomics (as the reference does), so
        # results agree to rounding, not bit for bit.
        for a, b in zip(pots, ref_p):
            assert np.max(np.abs(a - b)) <= 1e-13 * np.max(np.abs(b))
        for a, b in zip(forces, ref_f):
            assert np.max(np.abs(a - b)) <= 1e-13 * np.max(np.abs(b))
