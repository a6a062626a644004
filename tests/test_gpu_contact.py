"""Contact between materials against the oracle.

contacttype 0 (kernel contact): particles of other materials are appended to
the neighbour lists (MCM/mcm_ll_neighbours.f90:238-267).  contacttype > 0:
they form contact lists instead (:150-174), Monaghan's repulsive acceleration
over them (MCM/mcm_rep_contact.f90:37-161, called at mcm_solution.f90:64)
starts each particle's momentum sum (mcm_oldacceleration.f90:49-56,
mcm_corr_acceleration.f90:45-49), and the per-material contact forces sum
mass x repulsion for the time-history file.
"""
import numpy as np
import pytest

from mcmtop_b200 import _abi
from mcmtop_b200.deck import two_material_bar
from mcmtop_b200.solver import Solver
from oracle.pyoracle import Oracle
from test_gpu_parity import STATE, compare, compare_neighbours, relerr

pytestmark = pytest.mark.gpu


def compare_contacts(sol, orc):
    nc, cont, gc, gcont = sol.contacts()
    assert np.array_equal(nc, orc.get_int("ncont")), "contact counts differ"
    assert np.array_equal(gc, orc.get_int("g_ncont")), "ghost contact counts differ"
    for i in range(sol.n):
        assert np.array_equal(cont[i, : nc[i]], orc.contlist(i + 1)), f"contact sequence of particle {i + 1}"
        if gc[i]:
            assert np.array_equal(gcont[i, : gc[i]], orc.g_contlist(i + 1)), f"ghost contacts of particle {i + 1}"


@pytest.mark.parametrize("contacttype,disctype", [(0, 0), (1, 0), (1, 1)])
def test_contact_matches_oracle(contacttype, disctype, gpu_lib, oracle_lib):
    # FP64-exact: fields, accelerations, repulsion, lists and contact forces
    # after 30 steps, and each of the first steps' repulsion
    deck = two_material_bar(contacttype=contacttype, disctype=disctype)
    sol, orc = Solver(deck, _abi.PREC_FP64_EXACT), Oracle(deck)
    try:
        for k in range(30):
            sol.step()
            orc.step()
            if k < 3 and contacttype:
                assert relerr(sol.download(["repulsion"])["repulsion"], orc.get("repulsion")) <= 1e-12
        compare(sol, orc, STATE + ["a", "repulsion"], 1e-12, f"contacttype {contacttype}")
        compare_neighbours(sol, orc)
        if contacttype:
            # with kernel contact the reference's ncont counts the other
            # materials' particles, which the neighbour lists already hold
            compare_contacts(sol, orc)
        nn, nbr, gn, gnbr = sol.neighbours()
        mat = deck.mat
        cross = sum(int((mat[nbr[i, :nn[i]] - 1] != mat[i]).sum()) for i in range(deck.np))
        assert (cross == 0) == (contacttype > 0)
        cf, ocf = sol.contact_forces(), orc.contact_forces()
        if contacttype and disctype == 0:
            assert np.abs(ocf).max() > 0
            assert np.max(np.abs(cf - ocf)) <= 1e-12 * np.abs(ocf).max()
        else:
            assert not cf.any() and not ocf.any()
        assert relerr(sol.energies, orc.energies()) <= 1e-13
    finally:
        sol.close()
        orc.close()


@pytest.mark.parametrize("precision,tol", [(_abi.PREC_FP64, 1e-9), (_abi.PREC_MIXED, 5e-5)])
def test_contact_fast_paths(precision, tol, gpu_lib, oracle_lib):
    # the FP64-fast and mixed steps with repulsive contact against the oracle:
    # the same contact sets (sorted), fields within the precision's bound
    deck = two_material_bar(contacttype=1)
    sol, orc = Solver(deck, precision), Oracle(deck)
    try:
        for _ in range(20):
            sol.step()
            orc.step()
        compare(sol, orc, STATE + ["repulsion"], tol, f"precision {precision}")
        nc, cont, gc, gcont = sol.contacts()
        assert np.array_equal(nc, orc.get_int("ncont"))
        for i in range(0, deck.np, 7):
            assert np.array_equal(np.sort(cont[i, : nc[i]]), np.sort(orc.contlist(i + 1)))
    finally:
        sol.close()
        orc.close()


def test_repulsion_pushes_materials_apart(gpu_lib):
    # with contacttype 1 and K = 0 the halves pass through each other's
    # kernels without force; a positive K holds the upper half back
    a = Solver(two_material_bar(contacttype=1, k_cont=0.0), _abi.PREC_FP64)
    b = Solver(two_material_bar(contacttype=1, k_cont=1.0e-3), _abi.PREC_FP64)
    try:
        a.run(60)
        b.run(60)
        va, vb = a.download(["v"])["v"], b.download(["v"])["v"]
        upper = a.deck.mat == 2
        # the upper half moves along -z: the repulsion slows it
        assert vb[upper, 2].mean() > va[upper, 2].mean()
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("contacttype,kind", [(0, 2), (1, 2), (0, 3), (1, 3)])
def test_search_kinds_build_the_same_lists(contacttype, kind, gpu_lib):
    # one thread per particle against one warp per particle (2) or per cell
    # (3): same lists, same order, same ghosts, contacts and minimum distances
    # (FP64 exact path, a plane)
    deck = two_material_bar(contacttype=contacttype).replace(tcrit_opt=2)
    a, b = Solver(deck, _abi.PREC_FP64_EXACT), Solver(deck, _abi.PREC_FP64_EXACT)
    try:
        a.set_tuning(search_kind=1)
        b.set_tuning(search_kind=kind)
        assert a.tuning()["search_kind"] == 1 and b.tuning()["search_kind"] == kind
        for _ in range(5):
            a.step()
            b.step()
            for u, v in zip(a.neighbours(), b.neighbours()):
                assert np.array_equal(u, v)
            for u, v in zip(a.contacts(), b.contacts()):
                assert np.array_equal(u, v)
        sa, sb = a.download(STATE + ["mindist", "repulsion"]), b.download(STATE + ["mindist", "repulsion"])
        for f in sa:
            assert np.array_equal(sa[f], sb[f]), f
    finally:
        a.close()
        b.close()


def test_contact_list_regrow(gpu_lib, oracle_lib):
    # a contact list longer than its initial storage is regrown and the step
    # re-run, as for the neighbour table (MCM/mcm_ll_neighbours.f90:44,301-309)
    deck = two_material_bar(dx=0.6e-3, contacttype=1)
    sol, orc = Solver(deck, _abi.PREC_FP64_EXACT), Oracle(deck)
    try:
        for _ in range(3):
            sol.step()
            orc.step()
        nc = sol.contacts()[0]
        assert nc.max() > 16              # beyond the initial 16 entries per particle
        compare(sol, orc, STATE + ["repulsion"], 1e-12, "regrown contact lists")
    finally:
        sol.close()
        orc.close()


def test_time_history_contact_forces(tmp_path, gpu_lib, oracle_lib):
    # the _thist.csv columns of the contact forces come from the step's sums
    from mcmtop_b200.run import Program

    deck = two_material_bar(contacttype=1).replace(thpltime=0.0, stpltime=1.0e9, endtime=0.3)
    prog = Program(deck, "c", str(tmp_path), precision=_abi.PREC_FP64_EXACT)
    prog.initial()
    prog.run(max_steps=5)
    rows = [r for r in open(str(tmp_path / "c_thist.csv")).read().splitlines()[2:] if r.strip()]
    vals = np.array([[float(t) for t in r.split(",")[1:]] for r in rows])
    assert vals.shape[1] == 1 + 5 * 2
    assert not vals[0, 3:6].any()                    # initial row: no momentum sum yet
    assert np.abs(vals[1:, 5]).max() > 0             # zcf of material 1 after the first step
    prog.close()
