"""contacttype > 0: particles of other materials are not neighbours
(MCM/mcm_ll_neighbours.f90:238-267) and no contact force is added (the
reference's mcm_rep_cont has no call site), against the oracle."""
import dataclasses

import numpy as np
import pytest

from mcmtop_b200 import _abi
from mcmtop_b200.deck import taylor_bar
from mcmtop_b200.solver import Solver
from oracle.pyoracle import Oracle
from test_gpu_parity import STATE, compare, compare_neighbours

pytestmark = pytest.mark.gpu


def two_material_bar(contacttype):
    d = taylor_bar(dx=0.8e-3)
    upper = d.x[:, 2] > 0.5 * (d.x[:, 2].min() + d.x[:, 2].max())
    mat = np.where(upper, 2, 1).astype(np.int32)
    m1 = d.materials[0]
    dxc = 0.08
    mats = []
    for k, ys in ((1, 400e6), (2, 250e6)):
        m = dataclasses.replace(m1, strinput=m1.strinput.copy(), eosinput=m1.eosinput.copy())
        m.strinput[1] = ys * 1e-11
        m.mass = m.rho * int((mat == k).sum()) * dxc ** 3
        mats.append(m)
    return d.replace(materials=mats, mat=mat, contacttype=contacttype)


@pytest.mark.parametrize("contacttype", [0, 1])
def test_contact_type_matches_oracle(contacttype, gpu_lib, oracle_lib):
    deck = two_material_bar(contacttype)
    sol, orc = Solver(deck, _abi.PREC_FP64_EXACT), Oracle(deck)
    try:
        for _ in range(30):
            sol.step()
            orc.step()
        compare(sol, orc, STATE, 1e-12, f"contacttype {contacttype}")
        compare_neighbours(sol, orc)
        nn, nbr, gn, gnbr = sol.neighbours()
        mat = deck.mat
        cross = sum(int((mat[nbr[i, :nn[i]] - 1] != mat[i]).sum()) for i in range(deck.np))
        assert (cross == 0) == (contacttype > 0)
    finally:
        sol.close()
        orc.close()


def test_separate_materials_do_not_interact(gpu_lib):
    # with contacttype 1 the upper half cannot push the lower half: after the
    # impact wave the two halves separate where the kernel-contact bar does not
    a, b = Solver(two_material_bar(0), _abi.PREC_FP64), Solver(two_material_bar(1), _abi.PREC_FP64)
    try:
        a.run(60)
        b.run(60)
        va, vb = a.download(["v"])["v"], b.download(["v"])["v"]
        assert not np.array_equal(va, vb)
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("contacttype", [0, 1])
def test_search_kinds_build_the_same_lists(contacttype, gpu_lib):
    # one thread per particle and one warp per particle: same lists, same order,
    # same ghosts and minimum distances (FP64 exact path, two materials, a plane)
    deck = two_material_bar(contacttype).replace(tcrit_opt=2)
    a, b = Solver(deck, _abi.PREC_FP64_EXACT), Solver(deck, _abi.PREC_FP64_EXACT)
    try:
        a.set_tuning(search_kind=1)
        b.set_tuning(search_kind=2)
        assert a.tuning()["search_kind"] == 1 and b.tuning()["search_kind"] == 2
        for _ in range(5):
            a.step()
            b.step()
            la, lb = a.neighbours(), b.neighbours()
            for u, v in zip(la, lb):
                assert np.array_equal(u, v)
        sa, sb = a.download(STATE + ["mindist"]), b.download(STATE + ["mindist"])
        for f in sa:
            assert np.array_equal(sa[f], sb[f]), f
    finally:
        a.close()
        b.close()
