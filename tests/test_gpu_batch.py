"""Batched bodies (mcm_gpu_batch_*) and launch-shape tuning (mcm_gpu_autotune).

Neither changes the arithmetic of a body's step: a batch replays, as one CUDA
graph, the kernels mcm_gpu_run launches for each body, and a launch shape
only changes how particle groups are spread over blocks (each particle's sums
use the same 16 lanes in the same order).  So a body advanced in a batch, or
after tuning, must end bitwise where the same body advanced alone ends; only
the per-material energy sums, combined over a different number of block
partials, may differ in their last bits and are not compared.
"""
import numpy as np
import pytest

from mcmtop_b200 import _abi
from mcmtop_b200.deck import copper_model10, taylor_bar
from mcmtop_b200.solver import Batch, Solver

pytestmark = pytest.mark.gpu

STATE = ["x", "v", "rho", "e", "p", "c", "efps", "sigma", "q", "h"]
NSTEPS = 20


@pytest.fixture(scope="module")
def lib(gpu_lib):
    return gpu_lib


def bodies():
    """Five bars of different size, spacing, speed and yield stress."""
    out = []
    for k, (dx, r, ln, v, ys) in enumerate([(0.8e-3, 3.2e-3, 20e-3, 190.0, 400e6),
                                            (1.0e-3, 2.5e-3, 30e-3, 150.0, 300e6),
                                            (0.6e-3, 2.0e-3, 16e-3, 230.0, 550e6),
                                            (1.2e-3, 4.0e-3, 40e-3, 130.0, 250e6),
                                            (0.7e-3, 3.0e-3, 24e-3, 210.0, 450e6)]):
        mat = copper_model10(1.3 * dx * 100.0, yield_stress=ys)
        out.append(taylor_bar(dx=dx, radius=r, length=ln, velocity=v, seed=100 + k, material=mat))
    return out


def same_state(a: Solver, b: Solver):
    ga, gb = a.download(STATE), b.download(STATE)
    for f in STATE:
        assert np.array_equal(ga[f], gb[f]), f
    assert a.dt == b.dt and a.dtold == b.dtold and a.ptime == b.ptime


@pytest.mark.parametrize("precision", [_abi.PREC_FP64, _abi.PREC_MIXED, _abi.PREC_FP64_EXACT])
def test_batch_equals_individual_runs(lib, precision):
    decks = bodies()
    alone = [Solver(d, precision) for d in decks]
    for s in alone:
        assert s.run(NSTEPS) == NSTEPS
    together = [Solver(d, precision) for d in decks]
    batch = Batch(together, lanes=3)
    done = batch.run(12)
    done = done + batch.run(NSTEPS - 12)
    assert list(done) == [NSTEPS] * len(decks)
    for a, b in zip(alone, together):
        same_state(a, b)
    batch.close()


def test_batch_regrows_a_body_and_brings_it_level(lib):
    """A body whose neighbour table is too narrow overflows inside the graph;
    the batch regrows it, re-runs its remaining iterations alone, re-captures
    and goes on: the end state is the one of the body run alone."""
    decks = bodies()[:3]
    alone = [Solver(d, _abi.PREC_MIXED) for d in decks]
    for s in alone:
        s.run(NSTEPS)
    together = [Solver(d, _abi.PREC_MIXED) for d in decks]
    together[1].set_tuning(nbr_stride=8)
    batch = Batch(together, lanes=2)
    done = batch.run(NSTEPS)
    assert list(done) == [NSTEPS] * 3
    assert together[1].tuning()["nbr_stride"] > 8
    for a, b in zip(alone, together):
        same_state(a, b)
    batch.close()


def test_batch_termination_per_body(lib):
    decks = bodies()[:3]
    dt0 = Solver(decks[2], _abi.PREC_FP64).dt
    decks[2] = decks[2].replace(endtime=6.5 * dt0)
    alone = [Solver(d, _abi.PREC_FP64) for d in decks]
    n_alone = [s.run(NSTEPS) for s in alone]
    assert n_alone[2] < NSTEPS
    together = [Solver(d, _abi.PREC_FP64) for d in decks]
    batch = Batch(together, lanes=3)
    done = batch.run(NSTEPS)
    assert list(done) == n_alone
    for a, b in zip(alone, together):
        same_state(a, b)
    batch.close()


def test_autotune_keeps_state_and_results(lib):
    deck = bodies()[0]
    a = Solver(deck, _abi.PREC_MIXED)
    a.run(3)
    best = a.autotune(3)
    assert best["search_threads"] in (64, 128, 256) and best["pair_threads"] in (64, 128, 256)
    assert best["ms_per_step"] > 0.0 and best["nbr_stride"] >= a.stats()["max_nbr"]
    b = Solver(deck, _abi.PREC_MIXED)
    b.run(3)
    same_state(a, b)
    a.run(NSTEPS)
    b.run(NSTEPS)
    same_state(a, b)


@pytest.mark.parametrize("shape", [dict(search_threads=64, pair_threads=64, pair_blocks_per_sm=16),
                                   dict(search_threads=128, pair_threads=128, pair_blocks_per_sm=1),
                                   dict(search_threads=256, search_kind=2), dict(search_kind=3)])
def test_launch_shape_does_not_change_results(lib, shape):
    deck = bodies()[2]
    for precision in (_abi.PREC_FP64, _abi.PREC_MIXED):
        a = Solver(deck, precision)
        a.set_tuning(**shape)
        b = Solver(deck, precision)
        a.run(NSTEPS)
        b.run(NSTEPS)
        same_state(a, b)


def test_set_tuning_rejects_bad_shapes(lib):
    s = Solver(bodies()[0], _abi.PREC_MIXED)
    for bad in (dict(search_threads=96), dict(pair_threads=512), dict(pair_blocks_per_sm=17), dict(search_kind=4)):
        with pytest.raises(_abi.MCMError):
            s.set_tuning(**bad)


def test_batch_autotune_restores_states(lib):
    decks = bodies()
    alone = [Solver(d, _abi.PREC_MIXED) for d in decks]
    for s in alone:
        s.run(NSTEPS)
    together = [Solver(d, _abi.PREC_MIXED) for d in decks]
    batch = Batch(together, lanes=1)
    lanes, ms = batch.autotune(2)
    assert 1 <= lanes <= len(decks) and ms > 0.0
    batch.run(NSTEPS)
    for a, b in zip(alone, together):
        same_state(a, b)
    batch.close()


def _schedule(deck, nsteps):
    s = Solver(deck, _abi.PREC_FP64)
    out = [s.dt]
    for _ in range(nsteps):
        s.step_a()
        s.dt_update()
        out.append(s.dt)
        s.step_b()
        s.step_c()
    s.close()
    return np.array(out)


def _length_adjoint(x):
    xbar = np.zeros_like(x)
    xbar[int(x[:, 2].argmax()), 2] += 1.0
    xbar[int(x[:, 2].argmin()), 2] -= 1.0
    return xbar


def test_batched_adjoint_matches_each_body_alone(lib):
    """Gradients of the final bar length of every body of a batch
    (mcm_gpu_batch_adjoint_forward/backward, worker threads over the bodies)
    equal those of each body's own adjoint calls: parameter gradients and the
    initial-state adjoints.  Ghost-parent adjoints are summed with atomics, so
    the comparison allows the last bits (1e-12 relative)."""
    decks = bodies()
    nsteps, every = 24, 7
    dts = [_schedule(d, nsteps) for d in decks]
    batched = [Solver(d, _abi.PREC_FP64) for d in decks]
    batch = Batch(batched, lanes=3)
    batch.adjoint_forward(dts, every)
    xbars = [_length_adjoint(s.download(["x"])["x"]) for s in batched]
    pb, x0, v0 = batch.adjoint_backward(xbars, None)
    batch.close()
    for k, d in enumerate(decks):
        alone = Solver(d, _abi.PREC_FP64)
        alone.adjoint_forward(dts[k], every)
        xa = alone.download(["x"])["x"]
        assert np.array_equal(xa, batched[k].download(["x"])["x"]), k      # same forward, bitwise
        pa, xa0, va0 = alone.adjoint_backward(_length_adjoint(xa), None)
        alone.close()
        assert np.all(np.isfinite(pb[k])) and np.abs(pb[k]).max() > 0
        assert np.max(np.abs(pb[k] - pa)) <= 1e-12 * np.abs(pa).max(), (k, pb[k], pa)
        assert np.max(np.abs(x0[k] - xa0)) <= 1e-12 * np.abs(xa0).max(), k
        assert np.max(np.abs(v0[k] - va0)) <= 1e-12 * np.abs(va0).max(), k
    for s in batched:
        s.close()
