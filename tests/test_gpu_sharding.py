"""The multi-rank batched form on the CUDA library.

Two ranks (gloo process group, both on cuda:0: this checks the host logic and
the library path of each rank, not NVLink) split a set of independent cells by
sharding.shard_of, evaluate their shares with one batched library call each
(sharding.library_evaluator) and gather the results.  Every rank must end up
with every cell's potential and force, bitwise equal to a single-process
batched call on all cells: the evaluation is deterministic and a cell's result
does not depend on the other cells of its batch.
"""

import os
import socket

import numpy as np
import pytest

import workloads as W

pytestmark = pytest.mark.gpu


def _worker(rank, world, port, cells, tol, out_path):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    for p in (os.path.join(root, "dftb_fast-ewald_3d_b200"), here):
        sys.path.insert(0, p)
    import torch.distributed as dist

    import ewald_b200
    import sharding

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ctx = ewald_b200.Context(0, ewald_b200.FP64)
    try:
        mine = sharding.shard_of(cells, tol, sharding.library_parameters, rank, world)
        pots, forces = sharding.run_sharded(cells, tol, sharding.library_evaluator(ctx),
                                            sharding.library_parameters, rank, world)
        np.savez(out_path + f".{rank}.npz", np.asarray(mine), *pots, *forces)
    finally:
        ctx.close()
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_ranks_on_the_library_match_one_process_bitwise(tmp_path, ewald_lib):
    import torch.multiprocessing as mp

    cells = W.c4_batched_cells(12, seed=21)
    tol = 1e-10
    out = str(tmp_path / "res")
    mp.start_processes(_worker, args=(2, _free_port(), cells, tol, out), nprocs=2, join=True,
                       start_method="spawn")
    ctx = ewald_lib.Context(0, ewald_lib.FP64)
    try:
        ref_p, ref_f = ctx.batch_potential_force(cells, tol)
    finally:
        ctx.close()
    shards = []
    for rank in range(2):
        d = np.load(out + f".{rank}.npz")
        arrs = [d[f"arr_{i}"] for i in range(len(d.files))]
        shards.append(list(arrs[0]))
        pots, forces = arrs[1: 1 + len(cells)], arrs[1 + len(cells):]
        for a, b in zip(pots, ref_p):
            assert np.array_equal(a, b)
        for a, b in zip(forces, ref_f):
            assert np.array_equal(a, b)
    assert sorted(shards[0] + shards[1]) == list(range(len(cells)))
    assert shards[0] and shards[1]
