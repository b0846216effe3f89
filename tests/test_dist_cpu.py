"""Event sharding and max-over-ranks timing with two gloo ranks on the CPU (no GPU)."""
import os
import socket

import torch.multiprocessing as mp

from gvh import dist as gdist


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    r, w, local = gdist.rank_info()
    seed = gdist.event_seed(12345, r)
    ms = 10.0 + 5.0 * r          # rank 1 is the slow one
    ms_max = gdist.max_over_ranks(ms, dist, device="cpu")
    dist.barrier()
    out[rank] = (r, w, local, seed, ms_max, gdist.job_value(1000, 4, w, ms_max))
    dist.destroy_process_group()


def test_two_ranks_shard_events_and_take_the_slowest_time():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    assert sorted(out.keys()) == [0, 1]
    seeds = {out[r][3] for r in out.keys()}
    assert seeds == {12345, 12346}                     # one distinct event per rank
    for r in out.keys():
        rank, w, local, seed, ms_max, value = out[r]
        assert (rank, w, local) == (r, 2, r)
        assert ms_max == 15.0                          # the slowest rank's time on every rank
        assert value == 2 * 1000 * 4 / 0.015           # whole-job cell-updates/s


def test_single_process_defaults():
    assert gdist.rank_info() == (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                                 int(os.environ.get("LOCAL_RANK", "0")))
    assert gdist.max_over_ranks(3.5) == 3.5
    assert gdist.job_value(10, 2, 1, 1.0) == 20000.0
