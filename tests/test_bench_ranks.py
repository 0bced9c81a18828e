"""The benchmark's rank coordination with two ranks on the CPU (gloo): the
barrier, and the time every rank reports being the maximum over the ranks
(the rule for multi-GPU timings), as torchrun runs `bench.py --gpus 2`."""
import os
import sys

import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    torch.distributed.init_process_group('gloo', rank=rank, world_size=world)
    try:
        w, r, local = bench.dist_setup()
        assert (w, r, local) == (world, rank, rank)
        ranks = bench.Ranks(w, torch.device('cpu'))
        ranks.barrier()
        got = ranks.max(10.0 + 3.5 * rank)      # rank 1 is the slow one
        got1 = ranks.max(100.0 - rank)          # rank 0 is the slow one
        ranks.barrier()
        out[rank] = (got, got1)
    finally:
        torch.distributed.destroy_process_group()


def test_two_ranks_take_the_maximum_time():
    world = 2
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res == {0: (13.5, 100.0), 1: (13.5, 100.0)}


def test_one_rank_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    r = bench.Ranks(1, torch.device('cpu'))
    r.barrier()
    assert r.max(4.25) == 4.25
