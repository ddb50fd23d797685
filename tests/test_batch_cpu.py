"""Host-side logic of the batched solves (no GPU).

The batch workload's grid sizes are seeded and inside the stated corners; the
multi-rank split gives every system to exactly one rank, balanced by cells;
and the two-rank path of the batch benchmark (partition, max over ranks of the
device time, all-gather of per-rank statistics) runs on gloo.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from jxpamg_all_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_batch_grids_seeded_and_bounded():
    g1, g2 = synth.batch_grids(), synth.batch_grids()
    assert g1 == g2 and len(g1) == 64
    lo, hi = synth.BATCH_GRID_MIN, synth.BATCH_GRID_MAX
    for nx, ny, nz in g1:
        assert lo[0] <= nx <= hi[0] and lo[1] <= ny <= hi[1] and lo[2] <= nz <= hi[2]
    unknowns = 2 * sum(nx * ny * nz for nx, ny, nz in g1)
    assert 5_000_000 <= unknowns <= 20_000_000
    assert synth.batch_grids(size_seed=1) != g1


def test_batch_systems_small_sample():
    systems = synth.batch_systems(count=3, grid_max=(18, 18, 9))
    for k, s in enumerate(systems):
        assert s.block_size == 2 and s.n == 2 * s.nx * s.ny * s.nz
        # the diagonal block is the first entry of every row
        assert np.all(s.ja[s.ia[:-1]] == np.arange(s.num_block_rows))
    assert not np.array_equal(systems[0].b[:10], systems[1].b[:10])


@pytest.mark.parametrize("ws", [1, 2, 3, 8])
def test_batch_partition_complete_and_balanced(ws):
    sys.path.insert(0, ROOT)
    import bench

    cells = [nx * ny * nz for nx, ny, nz in synth.batch_grids()]
    parts = bench.batch_partition(cells, ws)
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(len(cells)))
    loads = [sum(cells[k] for k in p) for p in parts]
    assert max(loads) - min(loads) <= max(cells)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    cells = [nx * ny * nz for nx, ny, nz in synth.batch_grids()]
    mine = bench.batch_partition(cells, ws)[rank]
    t = torch.tensor([float(sum(cells[k] for k in mine))], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    stats = torch.tensor([float(len(mine)), float(sum(cells[k] for k in mine))], dtype=torch.float64)
    gathered = [torch.zeros_like(stats) for _ in range(ws)]
    dist.all_gather(gathered, stats)
    dist.barrier()
    dist.destroy_process_group()
    out[rank] = (float(t.item()), [g.tolist() for g in gathered], mine)


def test_batch_two_ranks_gloo():
    ws = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(ws, port, out), nprocs=ws, join=True)
        res = dict(out)
    cells = [nx * ny * nz for nx, ny, nz in synth.batch_grids()]
    mines = [res[r][2] for r in range(ws)]
    assert sorted(mines[0] + mines[1]) == list(range(64)) and not set(mines[0]) & set(mines[1])
    loads = [sum(cells[k] for k in m) for m in mines]
    for r in range(ws):
        assert res[r][0] == max(loads)
        assert [g[1] for g in res[r][1]] == loads
        assert int(sum(g[0] for g in res[r][1])) == 64
