"""Periodic boundary planes (MCM/mcm_init_boundary.f90:35-115, the wrap of
MCM/mcm_check_sym_pen.f90) and dynamic relaxation
(MCM/mcm_update_velocity.f90:33-44, MCM/mcm_write_drelax.f90) on the GPU
against the oracle."""
import numpy as np
import pytest

from mcmtop_b200 import _abi
from mcmtop_b200.deck import periodic_layer, taylor_bar
from mcmtop_b200.run import Program
from mcmtop_b200.solver import Solver
from oracle.pyoracle import Oracle
from test_gpu_parity import STATE, compare, compare_neighbours

pytestmark = pytest.mark.gpu


def test_periodic_planes_match_oracle(gpu_lib, oracle_lib):
    deck = periodic_layer(noise=2.0)
    sol, orc = Solver(deck, _abi.PREC_FP64_EXACT), Oracle(deck)
    try:
        x0 = deck.x.copy()
        for _ in range(60):
            sol.step()
            orc.step()
        compare(sol, orc, STATE, 1e-12, "periodic")
        compare_neighbours(sol, orc)
        par, gx, gv = sol.ghosts()
        assert len(par) == int(orc.scalar("ngp"))
        opar, ogx, ogv = orc.ghosts()
        assert np.array_equal(par, opar) and np.array_equal(gx, ogx)
        x = sol.download(["x"])["x"]
        assert (np.abs(x - x0) > 0.5 * (deck.sym_x[1] - deck.sym_x[0])).any()   # someone wrapped
    finally:
        sol.close()
        orc.close()


@pytest.mark.parametrize("prec,tol", [(_abi.PREC_FP64_EXACT, 1e-12), (_abi.PREC_MIXED, 2e-4)])
def test_dynamic_relaxation_matches_oracle(prec, tol, gpu_lib, oracle_lib):
    deck = taylor_bar(dx=0.8e-3).replace(drelax_scale=0.5)
    sol, orc = Solver(deck, prec), Oracle(deck)
    try:
        for _ in range(30):
            sol.step()
            orc.step()
        compare(sol, orc, ["x", "v", "rho", "p", "sigma", "vabs"], tol, "drelax")
    finally:
        sol.close()
        orc.close()


def test_relaxed_state_file(tmp_path, gpu_lib):
    deck = taylor_bar(dx=0.8e-3).replace(drelax_scale=0.5, endtime=0.2)
    p = Program(deck, "relax", str(tmp_path), _abi.PREC_FP64_EXACT)
    try:
        p.initial()
        p.run()
        p.finish()
        st = p.solver.download(["x", "mass", "h", "rho", "e"])
    finally:
        p.close()
    lines = (tmp_path / "relax.drlx").read_text().splitlines()
    assert lines[1] == "* Node Coordinates and Materials"
    node = lines[3:3 + deck.np]
    x = np.array([[float(ln[13 + 20 * k:33 + 20 * k]) for k in range(3)] for ln in node])
    np.testing.assert_allclose(x, st["x"], rtol=5e-13, atol=0)
    data = lines[3 + deck.np + 3:]
    assert len(data) == deck.np
    rho = np.array([float(ln[48:68]) for ln in data])
    np.testing.assert_allclose(rho, st["rho"], rtol=5e-13)
