"""The replica (view-sharded) multi-GPU path on CPU with two gloo ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from cindergs_b200.replicas import max_over_ranks, view_frames


def test_view_frames_partition():
    world, steps = 4, 7
    frames = [f for r in range(world) for f in view_frames(r, world, steps)]
    assert sorted(frames) == list(range(world * steps))
    with pytest.raises(ValueError):
        view_frames(4, 4, 1)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        frames = view_frames(rank, world, 5)
        elapsed = 10.0 + rank  # each rank's own "device time"
        out[rank] = (frames, max_over_ranks(elapsed))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_views_and_take_max_time():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0][1] == out[1][1] == 11.0
    assert set(out[0][0]).isdisjoint(out[1][0])
    assert sorted(out[0][0] + out[1][0]) == list(range(10))
