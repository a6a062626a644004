"""The multi-GPU host logic with two ranks on the CPU (gloo over 127.0.0.1):
the job's time is the slowest rank's, the job's rate counts every rank's
particles, and the ensemble blocks of the ranks cover every body once."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from mcmtop_b200.ranks import job_rate, share


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from mcmtop_b200.ranks import max_over_ranks

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        ms = 10.0 + 5.0 * rank                 # the second rank is slower
        out[rank] = max_over_ranks(ms, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    assert dict(out) == {0: 15.0, 1: 15.0}
    # 2 ranks x 2 034 720 particles x 100 steps in the slowest rank's 470 ms
    assert job_rate(2034720 * 100, 2, 470.0) == pytest.approx(2 * 2034720 * 100 / 0.47)


def test_max_without_a_process_group():
    from mcmtop_b200.ranks import max_over_ranks

    assert max_over_ranks(3.5) == 3.5


@pytest.mark.parametrize("n,world", [(256, 1), (256, 3), (5, 8), (0, 2), (257, 8)])
def test_ensemble_blocks_cover_every_body_once(n, world):
    seen = [i for r in range(world) for i in share(n, world, r)]
    assert seen == list(range(n))
    sizes = [len(share(n, world, r)) for r in range(world)]
    assert max(sizes) - min(sizes) <= 1
