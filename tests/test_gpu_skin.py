"""Skin lists (nbr_skin > 0) for the FP64-fast and mixed steps.

The neighbour lists of every step are filtered from a superset kept within
h_i + h_j + skin since the last build, which is redone when some particle has
moved half the skin.  The filter applies the search's own decisions to the
candidates of the 27 cells around each particle, so the neighbour SETS must be
the reference's at every step (their order is the skin list's, which only the
FP64-exact step would notice; that step keeps the full search).
"""
import numpy as np
import pytest

from mcmtop_b200 import _abi
from mcmtop_b200.deck import fluid_column, taylor_bar, two_material_bar
from mcmtop_b200.solver import Solver
from oracle.pyoracle import Oracle
from test_gpu_parity import STATE, compare, compare_neighbours

pytestmark = pytest.mark.gpu

SKIN = 0.3


def same_sets(sol, orc, contacts=False):
    compare_neighbours(sol, orc)   # sorted sets, ghosts by source and position
    if contacts:
        nc, cont, _, _ = sol.contacts()
        assert np.array_equal(nc, orc.get_int("ncont"))
        for i in range(sol.n):
            assert np.array_equal(np.sort(cont[i, : nc[i]]), np.sort(orc.contlist(i + 1))), f"contacts of {i + 1}"


@pytest.mark.parametrize("precision,tol", [(_abi.PREC_FP64, 1e-9), (_abi.PREC_MIXED, 5e-5)])
def test_skin_lists_give_the_reference_sets_every_step(precision, tol, gpu_lib, oracle_lib):
    deck = taylor_bar(dx=0.8e-3)
    sol, orc = Solver(deck, precision, nbr_skin=SKIN), Oracle(deck)
    try:
        for _ in range(60):
            sol.step()
            orc.step()
            same_sets(sol, orc)
        builds = sol.skin_builds()
        # the bar moves ~1.4 % of h per step: the skin of 0.3 h lasts several steps
        assert 2 <= builds <= 30, builds
        compare(sol, orc, STATE, tol, f"skin lists, precision {precision}")
    finally:
        sol.close()
        orc.close()


def test_skin_lists_with_ghost_walls_and_resorting(gpu_lib, oracle_lib):
    # five symmetry walls (ghosts of ghosts), gravity, particles re-sorted every
    # 4 steps (each re-sort forces a build: the lists hold state indices)
    deck = fluid_column(dx=0.01, block=(0.1, 0.06, 0.2), box=(0.4, 0.06, 0.3))
    sol = Solver(deck, _abi.PREC_MIXED, nbr_skin=SKIN, reorder_interval=4)
    orc = Oracle(deck)
    try:
        for _ in range(12):
            sol.step()
            orc.step()
            same_sets(sol, orc)
        assert sol.skin_builds() >= 3
        compare(sol, orc, STATE, 5e-5, "fluid column with skin lists")
    finally:
        sol.close()
        orc.close()


def test_skin_lists_with_contact(gpu_lib, oracle_lib):
    deck = two_material_bar(contacttype=1)
    sol, orc = Solver(deck, _abi.PREC_FP64, nbr_skin=SKIN), Oracle(deck)
    try:
        for _ in range(20):
            sol.step()
            orc.step()
            same_sets(sol, orc, contacts=True)
        compare(sol, orc, STATE + ["repulsion"], 1e-9, "contact with skin lists")
    finally:
        sol.close()
        orc.close()


def test_skin_fused_run_equals_split_steps(gpu_lib):
    deck = taylor_bar(dx=0.8e-3)
    a = Solver(deck, _abi.PREC_MIXED, nbr_skin=SKIN)
    b = Solver(deck, _abi.PREC_MIXED, nbr_skin=SKIN)
    try:
        for _ in range(25):
            a.step()
        assert b.run(25) == 25
        ga, gb = a.download(STATE), b.download(STATE)
        for f in STATE:
            assert np.array_equal(ga[f], gb[f]), f
        assert a.skin_builds() == b.skin_builds()
    finally:
        a.close()
        b.close()


def test_skin_lists_rejected_where_they_do_not_apply(gpu_lib):
    deck = taylor_bar(dx=0.8e-3)
    with pytest.raises(_abi.MCMError):
        Solver(deck, _abi.PREC_FP64_EXACT, nbr_skin=SKIN)      # keeps the reference's order
    with pytest.raises(_abi.MCMError):
        Solver(deck.replace(h_opt=1), _abi.PREC_FP64, nbr_skin=SKIN)   # h changes between builds
    s = Solver(deck, _abi.PREC_FP64, nbr_skin=SKIN)
    try:
        with pytest.raises(_abi.MCMError):
            s.adjoint_forward([s.dt] * 3, 2)
    finally:
        s.close()
