"""Multi-process host logic of bench.py on CPU with the gloo backend
(world_size 2): max-over-ranks timing and the rank-0-only reference arm."""

import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        got = bench.max_over_ranks(1.5 + rank, torch.device("cpu"))
        # the reference arm prints on rank 0 only; other ranks return 0 at once
        rc = bench.reference_arm(bench.parse_args(["--impl", "reference"])) if rank else None
        q.put((rank, got, rc))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_reference_arm_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(world))
    assert [r[1] for r in res] == [2.5, 2.5]
    assert res[1][2] == 0
