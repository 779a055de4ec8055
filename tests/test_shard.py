"""CPU: the multi-rank path for batches (trussnet_b200/shard.py) over gloo,
world size 2. Each rank relaxes its share with the CPU restatement (standing in
for the per-GPU relax_cl_batch); the gathered result must equal relaxing every
volume in one process, and the assignment must cover every volume once."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from trussnet_b200.shard import assign_volumes


def test_assignment_balanced_and_complete():
    counts = [5000, 400000, 120000, 9000, 300000, 77000, 5000, 250000]
    for world in (1, 2, 3, 4, 8):
        parts = assign_volumes(counts, world)
        flat = sorted(v for p in parts for v in p)
        assert flat == list(range(len(counts)))
        loads = [sum(counts[v] for v in p) for p in parts]
        # LPT: the heaviest rank carries at most 4/3 of the optimum (lower bound: max(mean, max item))
        lb = max(sum(counts) / world, max(counts))
        assert max(loads) <= 4 / 3 * lb + 1
    assert assign_volumes(counts, 3) == assign_volumes(list(counts), 3)


def _batch():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from trussnet_b200 import synth
    vols = [synth.sphere(dim=32, radius=10.0, seed=s) for s in range(3)]
    vols.append(synth.shells(dim=40, nshell=2, rmin=8.0, rmax=15.0, amp=1.0, hlo=1.5, hhi=3.0, density=1.0, seed=4))
    from trussnet_b200.types import RelaxParams
    prms = [RelaxParams(max_iters=15, dptol=0.0) for _ in vols]
    return vols, prms


def _oracle_relax(grids, prms, nodes, device):
    from oracle.oracle import Oracle
    o = Oracle("f32")
    return [o.relax(g, p, nd) for g, p, nd in zip(grids, prms, nodes)]


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from trussnet_b200.shard import relax_batch_distributed
        vols, prms = _batch()
        nodes = [nd.copy() for _, nd in vols]
        stats = relax_batch_distributed([g for g, _ in vols], prms, nodes, device=-1, relax_fn=_oracle_relax)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), *[nd.P for nd in nodes],
                 iters=np.array([s.iters for s in stats]))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_batch_equals_single_process(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    vols, prms = _batch()
    want = [nd.copy() for _, nd in vols]
    _oracle_relax([g for g, _ in vols], prms, want, -1)
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npz")
        for v, w in enumerate(want):
            assert np.array_equal(got[f"arr_{v}"].view(np.uint32), w.P.view(np.uint32)), (r, v)
        assert list(got["iters"]) == [15] * len(want)
