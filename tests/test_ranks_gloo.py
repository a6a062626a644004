"""The multi-GPU host logic with two ranks on the CPU (gloo over 127.0.0.1):
the job's time is the slowest rank's, the job's rate counts every rank's
particles, the ensemble blocks of the ranks cover every body once, and two
ranks that each advance their block of an ensemble (the CPU oracle standing
in for the GPU step) gather the same per-body results as one process that
advances every body."""
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


def _ensemble_decks():
    from mcmtop_b200.deck import taylor_bar

    # five small bars of different spacing, length and impact speed
    return [taylor_bar(dx=dx, radius=1.2e-3, length=L, velocity=v, seed=90 + k)
            for k, (dx, L, v) in enumerate([(0.5e-3, 6e-3, 150.0), (0.45e-3, 5e-3, 190.0), (0.6e-3, 8e-3, 220.0),
                                            (0.5e-3, 7e-3, 130.0), (0.55e-3, 6e-3, 240.0)])]


def _body_result(deck, steps):
    """Final length and the z-momentum of one bar after `steps` iterations of the oracle."""
    from oracle.pyoracle import Oracle

    orc = Oracle(deck)
    orc.run(steps)
    x, v, m = orc.get("x"), orc.get("v"), orc.get("mass")
    out = (float(x[:, 2].max() - x[:, 2].min()), float((m * v[:, 2]).sum()))
    orc.close()
    return out


def _ensemble_rank(rank, world, port, steps, out):
    import datetime

    import torch.distributed as dist

    from mcmtop_b200.ranks import gather_items, sum_over_ranks

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        decks = _ensemble_decks()
        mine = share(len(decks), world, rank)
        results = {k: _body_result(decks[k], steps) for k in mine}
        work = float(sum(decks[k].np * steps for k in mine))
        gathered = gather_items(results, len(decks), "cpu", width=2)
        total = sum_over_ranks(work, "cpu")
        out[rank] = (gathered.tolist(), total, list(mine))
    finally:
        dist.destroy_process_group()


def test_two_ranks_run_their_ensemble_blocks():
    steps = 6
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_ensemble_rank, args=(r, 2, port, steps, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    decks = _ensemble_decks()
    serial = [list(_body_result(d, steps)) for d in decks]
    g0, total0, mine0 = out[0]
    g1, total1, mine1 = out[1]
    assert mine0 == [0, 1, 2] and mine1 == [3, 4]
    assert g0 == g1 == serial                 # bitwise: the same oracle runs, gathered exactly
    assert total0 == total1 == sum(d.np * steps for d in decks)
