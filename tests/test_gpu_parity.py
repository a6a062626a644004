"""Parity of the CUDA step (through the C ABI) with the CPU oracle.

The FP64-exact flavour evaluates the reference's expressions in the
reference's order without fused multiply-add, and the neighbour search returns
the reference's neighbour sequences, so the fields agree to the last few bits
(transcendental functions such as tan and pow may differ by an ulp between the
CUDA and host math libraries).  Neighbour lists and ghosts are compared
exactly.  Tolerances are relative to the field's largest magnitude.
"""
import numpy as np
import pytest

from mcmtop_b200 import _abi
from mcmtop_b200.deck import fluid_column, taylor_bar
from mcmtop_b200.solver import Solver
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu

STATE = ["x", "v", "mass", "h", "rho", "e", "p", "c", "efps", "pcut", "fail", "vabs", "sigma", "q"]
DIAG = ["rod", "spin", "tracerod", "rhoold", "etry", "s"]


def relerr(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.max(np.abs(b)) if b.size else 0.0
    if scale == 0.0:
        return float(np.max(np.abs(a))) if a.size else 0.0
    return float(np.max(np.abs(a - b)) / scale)


def compare(sol, orc, fields, tol, label=""):
    g = sol.download(fields)
    worst = {}
    for f in fields:
        e = relerr(g[f], orc.get(f))
        worst[f] = e
    bad = {f: e for f, e in worst.items() if e > tol}
    assert not bad, f"{label} fields beyond {tol}: {bad}"
    return worst


def ghost_ids_as_oracle(sol, orc):
    """1-based oracle ghost id of each GPU ghost (index 0-based): the ghost of
    the same source particle at the nearest position.  The FP64-fast and mixed
    steps create their ghosts in their own cell order, so the ghost numbering
    differs from the reference's while the ghosts are the same."""
    gpar, gx, _ = sol.ghosts()
    opar, ox, _ = orc.ghosts()
    assert len(gpar) == len(opar), "ghost counts differ"
    assert np.array_equal(np.sort(gpar), np.sort(opar)), "ghost sources differ"
    by_par = {}
    for q, p in enumerate(opar):
        by_par.setdefault(int(p), []).append(q)
    out = np.empty(len(gpar), dtype=np.int64)
    for q, p in enumerate(gpar):
        cands = by_par[int(p)]
        d = [float(np.abs(ox[c] - gx[q]).max()) for c in cands]
        out[q] = cands[int(np.argmin(d))] + 1
    assert len(np.unique(out)) == len(out), "ghosts do not pair one to one"
    return out


def compare_neighbours(sol, orc):
    """The FP64-exact step's lists are the reference's sequences; the FP64-fast
    and mixed steps keep their cells in x order, so their lists hold the
    reference's sets (compared sorted, ghosts by source and position)."""
    ordered = sol.cfg.precision == _abi.PREC_FP64_EXACT
    key = (lambda v: v) if ordered else np.sort
    nn, nbr, gn, gnbr = sol.neighbours()
    onn = orc.get_int("nnbr")
    ogn = orc.get_int("g_nnbr")
    assert np.array_equal(nn, onn), "neighbour counts differ"
    assert np.array_equal(gn, ogn), "ghost neighbour counts differ"
    gmap = None if ordered or not gn.any() else ghost_ids_as_oracle(sol, orc)
    for i in range(sol.n):
        ref = orc.nbrlist(i + 1)
        assert np.array_equal(key(nbr[i, : nn[i]]), key(ref)), f"neighbour list of particle {i + 1} differs"
        if gn[i]:
            gref = orc.g_nbrlist(i + 1)
            got = gnbr[i, : gn[i]] if gmap is None else gmap[gnbr[i, : gn[i]] - 1]
            assert np.array_equal(key(got), key(gref)), f"ghost list of particle {i + 1} differs"


def small_bar(**kw):
    return taylor_bar(dx=0.8e-3, **kw)


@pytest.fixture(scope="module")
def lib(gpu_lib):
    return gpu_lib


def test_initial_state(lib):
    deck = small_bar()
    sol = Solver(deck, _abi.PREC_FP64_EXACT)
    orc = Oracle(deck)
    compare(sol, orc, STATE, 0.0, "initial")
    assert sol.dt == orc.scalar("dt")
    compare_neighbours(sol, orc)


def test_grid_and_ghosts(lib):
    deck = small_bar()
    sol = Solver(deck, _abi.PREC_FP64_EXACT)
    orc = Oracle(deck)
    gl, gm, gs = sol.grid()
    ogl, ogm, ogs = orc.grid()
    assert np.array_equal(gl, ogl) and np.array_equal(gm, ogm) and np.array_equal(gs, ogs)
    par, x, v = sol.ghosts()
    opar, ox, ov = orc.ghosts()
    assert len(par) == len(opar) > 0
    assert np.array_equal(par, opar)
    assert np.array_equal(x, ox) and np.array_equal(v, ov)


@pytest.mark.parametrize("disctype", [0, 1])
def test_one_step(lib, disctype):
    deck = small_bar(disctype=disctype)
    sol = Solver(deck, _abi.PREC_FP64_EXACT)
    orc = Oracle(deck)
    c_gpu = sol.step_a()
    c_orc = orc.step_a()
    assert abs(c_gpu - c_orc) <= 1e-15 * abs(c_orc)
    compare_neighbours(sol, orc)
    compare(sol, orc, STATE + DIAG, 1e-13, "after step_a")
    sol.dt_update()
    orc.dt_update()
    sol.step_b()
    orc.step_b()
    assert relerr(sol.energies, orc.energies()) < 1e-13
    compare(sol, orc, ["a"], 1e-12, "acceleration")
    sol.step_c(bbox=True)
    orc.step_c()
    compare(sol, orc, STATE, 1e-13, "after step_c")
    # mcm_coord_maxmin of MCM/mcm_move.f90:26-39 (before the plane checks)
    x = orc.get("x")
    assert np.allclose(sol.bbox[0::2], x.min(axis=0), rtol=0, atol=1e-9)
    assert np.allclose(sol.bbox[1::2], x.max(axis=0), rtol=0, atol=1e-9)


@pytest.mark.parametrize("disctype", [0, 1])
def test_twenty_steps(lib, disctype):
    deck = small_bar(disctype=disctype)
    sol = Solver(deck, _abi.PREC_FP64_EXACT)
    orc = Oracle(deck)
    for _ in range(20):
        sol.step()
        orc.step()
    assert abs(sol.ptime - orc.scalar("ptime")) <= 1e-12 * orc.scalar("ptime")
    compare(sol, orc, STATE, 1e-10, "20 steps")
    compare_neighbours(sol, orc)


def test_fused_run_equals_split(lib):
    deck = small_bar()
    a = Solver(deck, _abi.PREC_FP64_EXACT)
    b = Solver(deck, _abi.PREC_FP64_EXACT)
    for _ in range(15):
        a.step()
    done = b.run(15)
    assert done == 15
    assert a.dt == b.dt and a.ptime == b.ptime
    ga = a.download(STATE)
    gb = b.download(STATE)
    for f in STATE:
        assert np.array_equal(ga[f], gb[f]), f


def test_termination(lib):
    deck = small_bar()
    orc = Oracle(deck)
    dt0 = orc.scalar("dt")
    deck = deck.replace(endtime=5.5 * dt0)
    sol = Solver(deck, _abi.PREC_FP64_EXACT)
    orc = Oracle(deck)
    n_orc = orc.run(100)
    n_gpu = sol.run(100)
    assert n_gpu == n_orc
    compare(sol, orc, STATE, 1e-12, "terminated run")


@pytest.mark.parametrize("tcrit", [0, 2])
def test_timestep_options(lib, tcrit):
    deck = small_bar(tcrit_opt=tcrit)
    sol = Solver(deck, _abi.PREC_FP64_EXACT)
    orc = Oracle(deck)
    assert abs(sol.dt - orc.scalar("dt")) <= 1e-15 * orc.scalar("dt")
    for _ in range(3):
        sol.step()
        orc.step()
    compare(sol, orc, STATE, 1e-12, f"tcrit {tcrit}")


def test_fp64_fast(lib):
    deck = small_bar()
    sol = Solver(deck, _abi.PREC_FP64)
    orc = Oracle(deck)
    for _ in range(20):
        sol.step()
        orc.step()
    compare(sol, orc, STATE, 1e-9, "fp64 fast")
    compare_neighbours(sol, orc)


def test_fluid_column_five_planes(lib):
    deck = fluid_column(dx=0.01, block=(0.1, 0.06, 0.2), box=(0.4, 0.06, 0.3))
    sol = Solver(deck, _abi.PREC_FP64_EXACT)
    orc = Oracle(deck)
    par, x, v = sol.ghosts()
    opar, ox, ov = orc.ghosts()
    assert np.array_equal(par, opar) and np.array_equal(x, ox)
    compare_neighbours(sol, orc)
    for _ in range(10):
        sol.step()
        orc.step()
    compare(sol, orc, STATE, 1e-10, "fluid")
    compare_neighbours(sol, orc)


@pytest.mark.parametrize("disctype", [0, 1])
def test_taylor_bar_16k_steps(lib, disctype):
    """The 16 848-particle Taylor bar (dx = 0.4 mm), first 30 steps, simple and
    corrected SPH."""
    deck = taylor_bar(dx=0.4e-3, disctype=disctype)
    assert deck.np == 16848
    sol = Solver(deck, _abi.PREC_FP64_EXACT)
    orc = Oracle(deck, openmp=True)
    for _ in range(30):
        sol.step()
        orc.step()
    compare(sol, orc, STATE, 1e-10, "16k bar")
    compare_neighbours(sol, orc)


def test_taylor_bar_16k_thousand_steps(lib):
    """The 16 848-particle bar for the 1000 steps of its configuration: the
    FP64-exact step against the oracle (OpenMP build) at the end, through the
    fused device loop.  The per-step differences (transcendentals an ulp
    apart) grow over the run; the bound is 1e-8 of each field's range."""
    deck = taylor_bar(dx=0.4e-3)
    sol = Solver(deck, _abi.PREC_FP64_EXACT)
    orc = Oracle(deck, openmp=True)
    # the total-energy balance of mcm_calctotale (MCM/mcm_calctotale.f90:53-60)
    # along the run: the GPU's drift follows the oracle's every 100 steps
    e0, o0 = sol.energies_now()[-1], orc.scalar("totale")
    # block partials against the oracle's serial sum over 16 848 particles
    assert abs(e0 - o0) <= 1e-11 * abs(o0)
    for _ in range(10):
        assert sol.run(100) == 100
        assert orc.run(100) == 100
        drift_gpu = (sol.energies_now()[-1] - e0) / e0
        drift_orc = (orc.scalar("totale") - o0) / o0
        assert abs(drift_gpu - drift_orc) <= 1e-9, (drift_gpu, drift_orc)
    errs = compare(sol, orc, STATE, 1e-8, "16k bar, 1000 steps")
    print("max relative error per field after 1000 steps:", errs, "energy drift", drift_orc)
    assert abs(sol.ptime - orc.scalar("ptime")) <= 1e-10 * orc.scalar("ptime")


def test_displacement_bcs(lib, oracle_lib):
    """Displacement codes 1-7 (MCM/mcm_boundcond.f90:30-61 zero the
    constrained acceleration components; MCM/mcm_init_boundcond.f90:25-54
    zero the constrained initial velocity components) on a bar whose
    particles carry seeded random codes, against the oracle in all three
    precisions; constrained velocity components stay zero."""
    deck = small_bar()
    rng = np.random.default_rng(11)
    deck = deck.replace(dispbc=rng.integers(0, 8, size=deck.np).astype(np.int32))
    masks = {1: (1, 0, 0), 2: (0, 1, 0), 3: (0, 0, 1), 4: (1, 1, 0), 5: (0, 1, 1), 6: (1, 0, 1), 7: (1, 1, 1)}
    for prec, tol in ((_abi.PREC_FP64_EXACT, 1e-12), (_abi.PREC_FP64, 1e-9), (_abi.PREC_MIXED, 5e-5)):
        sol, orc = Solver(deck, prec), Oracle(deck)
        try:
            for _ in range(25):
                sol.step()
                orc.step()
            compare(sol, orc, STATE + ["a"], tol, f"dispbc, precision {prec}")
            v = sol.download(["v"])["v"]
            for code, m in masks.items():
                sel = deck.dispbc == code
                for d in range(3):
                    if m[d]:
                        assert not v[sel, d].any(), (code, d)
        finally:
            sol.close()
            orc.close()


def test_neighbour_overflow_regrow(lib):
    """A too narrow initial table is regrown and the step re-run."""
    deck = small_bar()
    sol = Solver(deck, _abi.PREC_FP64_EXACT, nbr_stride=8)
    orc = Oracle(deck)
    compare_neighbours(sol, orc)
    sol.step()
    orc.step()
    compare(sol, orc, STATE, 1e-12, "after regrow")
    assert sol.stats()["stride"] >= orc.get_int("nnbr").max()


@pytest.mark.parametrize("disctype", [0, 1])
def test_reordering_does_not_change_results(lib, disctype):
    """Re-sorting the particle storage every 3 steps gives bitwise the same state."""
    deck = small_bar(disctype=disctype)
    a = Solver(deck, _abi.PREC_FP64_EXACT)
    b = Solver(deck, _abi.PREC_FP64_EXACT, reorder_interval=3)
    orc = Oracle(deck)
    for _ in range(10):
        a.step()
        b.step()
        orc.step()
    ga = a.download(STATE)
    gb = b.download(STATE)
    for f in STATE:
        assert np.array_equal(ga[f], gb[f]), f
    compare_neighbours(b, orc)


@pytest.mark.parametrize("precision", [_abi.PREC_FP64_EXACT, _abi.PREC_MIXED])
def test_search_prefilter_without_diagnostics(lib, precision):
    """With diagnostics off (and tcrit_opt 1) the search accepts clear
    neighbours from the FP32 test alone; the sets must still be the oracle's."""
    deck = taylor_bar(dx=0.4e-3)
    sol = Solver(deck, precision)
    sol.set_diagnostics(False)
    orc = Oracle(deck, openmp=True)
    for _ in range(5):
        sol.step()
        orc.step()
    if precision == _abi.PREC_FP64_EXACT:
        compare(sol, orc, STATE, 1e-11, "prefiltered search")
    compare_neighbours(sol, orc)


@pytest.mark.parametrize("kind", [2, 3])
def test_search_kinds_match_oracle(lib, kind):
    """The warp-per-particle and warp-per-cell searches build the reference's
    neighbour sequences on the fluid column (five ghost planes, ghosts of
    ghosts) and the 16 848-particle bar, with diagnostics off (FP32 decisions
    with FP64 ties only) and on (FP64 minimum distances)."""
    for deck in (fluid_column(dx=0.01, block=(0.1, 0.06, 0.2), box=(0.4, 0.06, 0.3)), taylor_bar(dx=0.4e-3)):
        for diag in (False, True):
            sol = Solver(deck, _abi.PREC_FP64_EXACT)
            sol.set_tuning(search_kind=kind)
            sol.set_diagnostics(diag)
            orc = Oracle(deck, openmp=True)
            for _ in range(3):
                sol.step()
                orc.step()
            compare_neighbours(sol, orc)
            compare(sol, orc, STATE + (["mindist"] if diag else []), 1e-12, f"search kind {kind}")
            sol.close()
            orc.close()
