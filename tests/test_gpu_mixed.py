"""Accuracy of the mixed-precision step against the FP64 oracle.

The mixed path computes the strain-rate and momentum pair sums in FP32 on
cell-relative positions: each of a particle's two lanes adds its half of the
terms plainly, and the two lane sums are combined by an error-free TwoSum and
rounded once to FP64; every per-particle field, the constitutive update, the
integration and the energy/timestep reductions stay FP64.  The neighbour
search is the exact FP64 one, so neighbour sets match the oracle's.  Field
errors are relative to each field's largest magnitude; the bound 2e-5 after
20 steps is about 100 FP32 ulps of the largest value.
"""
import numpy as np
import pytest

from mcmtop_b200 import _abi
from mcmtop_b200.deck import fluid_column, taylor_bar
from mcmtop_b200.solver import Solver
from oracle.pyoracle import Oracle

from test_gpu_parity import STATE, compare, compare_neighbours, relerr

pytestmark = pytest.mark.gpu

MIXED_TOL = 2e-5


@pytest.fixture(scope="module")
def lib(gpu_lib):
    return gpu_lib


def test_mixed_initial_state(lib):
    deck = taylor_bar(dx=0.8e-3)
    sol = Solver(deck, _abi.PREC_MIXED)
    orc = Oracle(deck)
    # initialisation is the FP64 one
    compare(sol, orc, STATE, 1e-14, "initial")
    assert abs(sol.dt - orc.scalar("dt")) <= 1e-14 * orc.scalar("dt")
    compare_neighbours(sol, orc)


def test_mixed_one_step_split(lib):
    deck = taylor_bar(dx=0.8e-3)
    sol = Solver(deck, _abi.PREC_MIXED)
    orc = Oracle(deck)
    c_gpu = sol.step_a()
    c_orc = orc.step_a()
    assert abs(c_gpu - c_orc) <= 1e-6 * abs(c_orc)
    compare_neighbours(sol, orc)
    compare(sol, orc, STATE + ["rod", "spin"], MIXED_TOL, "mixed step_a")
    sol.dt_update()
    orc.dt_update()
    sol.step_b()
    orc.step_b()
    assert relerr(sol.energies, orc.energies()) < 1e-6
    compare(sol, orc, ["a"], 1e-4, "mixed acceleration")
    sol.step_c()
    orc.step_c()
    compare(sol, orc, STATE, MIXED_TOL, "mixed step_c")


def test_mixed_twenty_steps(lib):
    deck = taylor_bar(dx=0.8e-3)
    sol = Solver(deck, _abi.PREC_MIXED)
    orc = Oracle(deck)
    for _ in range(20):
        sol.step()
        orc.step()
    assert abs(sol.ptime - orc.scalar("ptime")) <= 1e-6 * orc.scalar("ptime")
    compare(sol, orc, STATE, MIXED_TOL, "mixed 20 steps")


def test_mixed_fused_run_matches_split(lib):
    deck = taylor_bar(dx=0.8e-3)
    a = Solver(deck, _abi.PREC_MIXED)
    b = Solver(deck, _abi.PREC_MIXED)
    for _ in range(10):
        a.step()
    assert b.run(10) == 10
    ga = a.download(STATE)
    gb = b.download(STATE)
    for f in STATE:
        assert relerr(gb[f], ga[f]) <= 1e-6, f


def test_mixed_reordering(lib):
    """Re-sorting the storage leaves the mixed results bitwise unchanged (the
    gather records and the summation order follow the cell order)."""
    deck = taylor_bar(dx=0.8e-3)
    a = Solver(deck, _abi.PREC_MIXED)
    b = Solver(deck, _abi.PREC_MIXED, reorder_interval=3)
    for _ in range(10):
        a.step()
        b.step()
    ga = a.download(STATE)
    gb = b.download(STATE)
    for f in STATE:
        assert np.array_equal(ga[f], gb[f]), f


def test_mixed_fluid_column_ghosts(lib):
    """Ghost pairs (FP64 positions) in a water column with five planes."""
    deck = fluid_column(dx=0.01, block=(0.1, 0.06, 0.2), box=(0.4, 0.06, 0.3))
    sol = Solver(deck, _abi.PREC_MIXED)
    orc = Oracle(deck)
    for _ in range(10):
        sol.step()
        orc.step()
    compare(sol, orc, STATE, 1e-4, "mixed fluid")


def test_mixed_taylor_bar_16k(lib):
    deck = taylor_bar(dx=0.4e-3)
    sol = Solver(deck, _abi.PREC_MIXED)
    orc = Oracle(deck, openmp=True)
    for _ in range(30):
        sol.step()
        orc.step()
    compare(sol, orc, STATE, 1e-4, "mixed 16k bar")


def test_mixed_rejects_corrected_sph(lib):
    deck = taylor_bar(dx=0.8e-3, disctype=1)
    with pytest.raises(_abi.MCMError):
        Solver(deck, _abi.PREC_MIXED)


def test_mixed_energy_balance_16k_thousand_steps(lib):
    """The 16 848-particle bar for its 1000 steps in mixed precision.

    Every field stays within 1e-4 of its range of the FP64 oracle's over the
    first 400 steps: the physical time that the 2000 steps of the 2 034 720-
    particle bar (dx 0.08 mm, a time step 5x shorter) cover.  Beyond that the
    plastic front amplifies the FP32 rounding of the pair sums: the largest
    per-particle difference reaches about 2.5e-3 of the stress range at step
    1000 on a few hundred of the 16 848 particles, while the root-mean-square
    difference stays below 1e-4 of each field's range and the total energy of
    mcm_calctotale (MCM/mcm_calctotale.f90:53-60) drifts as the oracle's does
    (within 1e-5 of the initial total at every 100th step)."""
    deck = taylor_bar(dx=0.4e-3)
    sol = Solver(deck, _abi.PREC_MIXED)
    orc = Oracle(deck, openmp=True)
    e0, o0 = sol.energies_now()[-1], orc.scalar("totale")
    worst = 0.0
    for k in range(10):
        assert sol.run(100) == 100
        assert orc.run(100) == 100
        drift_gpu = (sol.energies_now()[-1] - e0) / e0
        drift_orc = (orc.scalar("totale") - o0) / o0
        worst = max(worst, abs(drift_gpu - drift_orc))
        if k < 4:
            compare(sol, orc, STATE, 1e-4, f"mixed 16k bar, {100 * (k + 1)} steps")
    assert worst <= 1e-5, worst
    g = sol.download(STATE)
    rms, mx = {}, {}
    for f in STATE:
        ref = orc.get(f)
        scale = float(np.max(np.abs(ref))) or 1.0
        d = np.abs(g[f] - ref)
        rms[f] = float(np.sqrt(np.mean(d ** 2))) / scale
        mx[f] = float(d.max()) / scale
    print("mixed, 1000 steps: energy drift gap", worst, "max", mx, "rms", rms)
    assert max(rms.values()) <= 1e-4, rms
    assert max(mx.values()) <= 1e-2, mx


def test_mixed_compensated_sums(lib):
    """The Kahan-compensated variant of the pair sums (compensated_sums): the
    same neighbour sets, fields within the mixed bound of the oracle after 20
    steps, and no further from it than the plain sums' worst field."""
    deck = taylor_bar(dx=0.8e-3)
    orc = Oracle(deck)
    plain, comp = Solver(deck, _abi.PREC_MIXED), Solver(deck, _abi.PREC_MIXED, compensated=True)
    for _ in range(20):
        plain.step()
        comp.step()
        orc.step()
    compare_neighbours(comp, orc)
    e_comp = compare(comp, orc, STATE, MIXED_TOL, "compensated mixed sums")
    e_plain = compare(plain, orc, STATE, MIXED_TOL, "plain mixed sums")
    print("worst field: compensated", max(e_comp.values()), "plain", max(e_plain.values()))
    assert max(e_comp.values()) <= 1.5 * max(e_plain.values())
    plain.close()
    comp.close()


def test_mixed_staged_strain_gather_is_bitwise_the_same(lib):
    """The strain and momentum gathers with each block's rows of neighbour
    records staged in shared memory (pair_kind 2) read the same records:
    bitwise the same state as the per-neighbour gathers, on the bar and on the
    fluid column (ghosts)."""
    for deck in (taylor_bar(dx=0.4e-3), fluid_column(dx=0.01, block=(0.1, 0.06, 0.2), box=(0.4, 0.06, 0.3))):
        a, b = Solver(deck, _abi.PREC_MIXED), Solver(deck, _abi.PREC_MIXED)
        b.set_tuning(pair_kind=2)
        assert b.tuning()["pair_kind"] == 2
        a.run(12)
        b.run(12)
        ga, gb = a.download(STATE), b.download(STATE)
        for f in STATE:
            assert np.array_equal(ga[f], gb[f]), f
        a.close()
        b.close()


def test_mixed_fluid_column_long_run(lib):
    """The column collapse (null material, EOS 1, gravity, five ghost walls)
    for 300 mixed-precision steps, the neighbour lists rebuilt every step:
    positions and velocities within 1e-4 of their range of the FP64 oracle's,
    the same neighbour sets at the end, and the total energy of mcm_calctotale
    within 1e-4 of the oracle's (relative to the largest kinetic energy)."""
    deck = fluid_column(dx=0.01, block=(0.1, 0.06, 0.2), box=(0.4, 0.06, 0.3))
    sol = Solver(deck, _abi.PREC_MIXED)
    orc = Oracle(deck)
    # the column starts at rest with zero internal energy: the totals are
    # compared against the largest kinetic energy the oracle reaches
    gaps, scale = [], 0.0
    for _ in range(6):
        assert sol.run(50) == 50
        assert orc.run(50) == 50
        gaps.append(abs(sol.energies_now()[-1] - orc.scalar("totale")))
        scale = max(scale, abs(orc.scalar("kinetice")))
    assert scale > 0.0
    gap = max(gaps) / scale
    assert gap <= 1e-4, gap
    errs = compare(sol, orc, ["x", "v"], 1e-4, "mixed fluid column, 300 steps")
    print("fluid column, 300 mixed steps:", errs, "energy gap", gap)
    nn, nbr, gn, gnbr = sol.neighbours()
    assert np.array_equal(nn, orc.get_int("nnbr"))
    for i in range(0, deck.np, 11):
        assert np.array_equal(np.sort(nbr[i, : nn[i]]), np.sort(orc.nbrlist(i + 1)))


def test_mixed_search_lists_without_diagnostics(lib):
    """With diagnostics off (one material, tcrit_opt 1) the mixed step's search
    takes its windowed loop whose accept path is a predicated store; with
    diagnostics on (FP64 minimum distances) it takes the branching loop.  The two must build the same lists, entry for entry, and
    the sets must be the oracle's, on the bar, on the fluid column (ghost
    walls, ghosts of ghosts) and on a bar with variable h, with the storage
    re-sorted every three steps."""
    decks = (taylor_bar(dx=0.4e-3), fluid_column(dx=0.01, block=(0.1, 0.06, 0.2), box=(0.4, 0.06, 0.3)),
             taylor_bar(dx=0.8e-3).replace(h_opt=2))   # h varies after the first step
    for deck in decks:
        a = Solver(deck, _abi.PREC_MIXED, reorder_interval=3)
        b = Solver(deck, _abi.PREC_MIXED, reorder_interval=3)
        a.set_diagnostics(False)
        b.set_diagnostics(True)
        # with variable h the mixed densities move h off the oracle's by FP32
        # amounts, so only the two GPU walks are compared there
        orc = Oracle(deck, openmp=True) if not deck.h_opt else None
        for _ in range(7):
            a.step()
            b.step()
            if orc:
                orc.step()
            na, la, gna, gla = a.neighbours()
            nb, lb, gnb, glb = b.neighbours()
            assert np.array_equal(na, nb) and np.array_equal(gna, gnb)
            w = int(na.max())
            m = np.arange(w)[None, :] < na[:, None]
            assert np.array_equal(la[:, :w][m], lb[:, :w][m])
        if orc:
            compare_neighbours(a, orc)
            orc.close()
        for f in STATE:
            assert np.array_equal(a.download([f])[f], b.download([f])[f]), f
        a.close()
        b.close()
