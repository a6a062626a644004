"""The cap model (model 4, MCM/mcm_f3dm25.f90) on the oracle and on the GPU.

The soil deck is a sand bar (mcmtop_b200.deck.sand_model4) in mm-ms-g units,
where stresses are in MPa: the model's absolute tolerances assume stresses of
order 1-100.  At 60 m/s the bar's particles go through the elastic mode (1),
the tension cut-off (2), the failure surface (4, 9, 10) and the cap (11).

The reference writes only the upper triangle of sigma in this model; the
lower triangle keeps the rotated stress, and the next rotation and the
momentum sum read it.  The GPU step supports the model with simple SPH in all
three precisions, whose momentum sums read both triangles; corrected SPH
(whose sum carries six components) reports it unsupported.  The model's own
arithmetic is single precision (undeclared Fortran locals), evaluated
identically on the oracle and the FP64-exact path (IEEE float operations
without contraction, exp as the rounded double exp); the FP64-fast and mixed
paths contract its float expressions, so a particle near a mode boundary can
take the other mode.
"""
import ctypes as C

import numpy as np
import pytest

from mcmtop_b200 import _abi
from mcmtop_b200.deck import MMMSG, sand_model4, taylor_bar
from oracle.pyoracle import Oracle

NSTEPS = 20
STATE = ["x", "v", "rho", "e", "p", "sigma", "q", "capa"]


def sand_bar(iterate=False, velocity=60.0):
    return taylor_bar(dx=0.8e-3, velocity=velocity, material=sand_model4(0.0, iterate=iterate), units=MMMSG)


def relerr(a, b):
    scale = float(np.max(np.abs(b)))
    return float(np.max(np.abs(a - b)) / scale) if scale > 0 else float(np.max(np.abs(a)))


# ------------------------------------------------------------------ CPU
def test_initial_cap_and_tension_cutoff():
    """mcm_sets4's initel: X0 = kappa0 + R Fe(kappa0) and Fe(fcut) = 0, to its
    absolute tolerance 1e-3 (MPa here)."""
    deck = sand_bar()
    orc = Oracle(deck)
    si, _, g = orc.material_table(1)
    cm = lambda i, j: si[(i - 1) + 5 * (j - 1)]   # noqa: E731
    alpha, theta, gama, beta, r = cm(1, 3), cm(1, 4), cm(1, 5), cm(1, 6), cm(2, 1)
    fe = lambda x: alpha - gama * np.exp(-beta * x) + theta * x   # noqa: E731
    k0, fcut = cm(3, 3), cm(3, 4)
    assert abs(cm(2, 5) - k0 - r * fe(k0)) <= 1e-3 and k0 > 0
    assert abs(fe(fcut)) <= 1e-3 and fcut < 0
    K, G = cm(1, 1), cm(1, 2)
    assert abs(cm(5, 2) - (K + 4.0 * G / 3.0)) <= 1e-9 * cm(5, 2)   # lambda + 2 mu
    assert g == G
    # initial state: at rest, p = 0, c = sqrt(cm(5,2)/rho0) (MCM/mcm_calcrhopc.f90:57-67)
    assert np.all(orc.get("p") == 0.0)
    assert np.allclose(orc.get("c"), np.sqrt(cm(5, 2) / deck.materials[0].rho), rtol=1e-15)


def test_oracle_soil_bar_visits_the_modes():
    deck = sand_bar()
    orc = Oracle(deck)
    seen = set()
    for _ in range(30):
        orc.step()
        seen |= set(np.unique(orc.get_int("ptype")).tolist())
    for f in STATE:
        assert np.all(np.isfinite(orc.get(f))), f
    assert {1, 10, 11} <= seen, seen
    assert np.max(orc.get("capa")) > sand_model4(0.0).strinput[12]   # the cap has moved
    # the lower triangle of sigma differs from the upper one only where the return map acted
    sig = orc.get("sigma")
    assert np.max(np.abs(sig[:, 0, 1] - sig[:, 1, 0])) > 0.0


def test_oracle_iterated_return_does_not_converge():
    """With the vector flag set (cm(3,5) /= 0) the returns iterate to |f| <= 1e-8,
    below single-precision resolution for stresses of this size: the reference
    stops ('feit1'/'fcit1'), the oracle reports MCM_ECAP_NOCONV."""
    orc = Oracle(sand_bar(iterate=True))
    with pytest.raises(RuntimeError, match="status 4"):
        for _ in range(5):
            orc.step()


def _lib_material(lib, card):
    m = _abi.Material()
    m.model, m.eos, m.visc_type = card.model, card.eos, card.visc_type
    m.rho, m.av_l, m.av_q, m.mass, m.h = card.rho, card.av_l, card.av_q, card.mass, card.h
    for i in range(48):
        m.strinput[i] = float(card.strinput[i])
    for i in range(24):
        m.eosinput[i] = float(card.eosinput[i])
    return lib.mcm_gpu_material_from_deck(C.byref(m)), m


def test_library_material_setup_matches_oracle():
    lib = _abi.load()
    deck = sand_bar()
    st, m = _lib_material(lib, deck.materials[0])
    assert st == _abi.MCM_OK
    si, ei, g = Oracle(deck).material_table(1)
    assert np.array_equal(np.array(m.strinput[:]), si)
    assert m.g == g
    bad = sand_model4(0.0)
    bad.strinput[26] = 3.0   # ltype outside {1, 2}
    assert _lib_material(lib, bad)[0] == _abi.MCM_EINVAL
    eos = sand_model4(0.0)
    eos.eos = 41
    assert _lib_material(lib, eos)[0] == _abi.MCM_EINVAL


@pytest.mark.parametrize("precision,disctype", [(_abi.PREC_FP64, 1), (_abi.PREC_FP64_EXACT, 1)])
def test_library_rejects_cap_model_with_corrected_sph(precision, disctype):
    from mcmtop_b200.solver import config_from_deck, material_table

    lib = _abi.load()
    deck = sand_bar().replace(disctype=disctype)
    cfg = config_from_deck(deck, precision)
    h = C.c_void_p()
    st = lib.mcm_gpu_create(C.byref(cfg), material_table(deck), 1, deck.np, C.byref(h))
    assert st == _abi.MCM_EUNSUPPORTED


# ------------------------------------------------------------------ GPU
@pytest.mark.gpu
def test_cap_model_parity_exact(gpu_lib):
    from mcmtop_b200.solver import Solver

    deck = sand_bar()
    sol = Solver(deck, _abi.PREC_FP64_EXACT)
    orc = Oracle(deck)
    for k in range(NSTEPS):
        sol.step()
        orc.step()
    got = sol.download(STATE + ["ptype"])
    assert np.array_equal(got["ptype"], orc.get_int("ptype"))
    errs = {f: relerr(got[f], orc.get(f)) for f in STATE}
    bad = {f: e for f, e in errs.items() if e > 1e-9}
    assert not bad, errs
    sig = got["sigma"]
    assert np.max(np.abs(sig[:, 0, 1] - sig[:, 1, 0])) > 0.0   # the asymmetric stress is carried
    sol.close()


@pytest.mark.gpu
def test_cap_model_iterated_return_reports_status(gpu_lib):
    from mcmtop_b200.solver import Solver

    sol = Solver(sand_bar(iterate=True), _abi.PREC_FP64_EXACT)
    with pytest.raises(_abi.MCMError) as e:
        for _ in range(5):
            sol.step()
    assert e.value.code == _abi.MCM_ECAP_NOCONV
    sol.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [(_abi.PREC_FP64, 1e-4), (_abi.PREC_MIXED, 2e-4)])
def test_cap_model_fast_and_mixed(gpu_lib, precision, tol):
    """The sand bar on the FP64-fast and mixed steps against the oracle: the
    same modes for all but a few particles near a mode boundary, every field
    within tol of its range, and the asymmetric stress carried."""
    from mcmtop_b200.solver import Solver

    deck = sand_bar()
    sol = Solver(deck, precision)
    orc = Oracle(deck)
    for _ in range(NSTEPS):
        sol.step()
        orc.step()
    got = sol.download(STATE + ["ptype"])
    differ = int(np.count_nonzero(got["ptype"] != orc.get_int("ptype")))
    assert differ <= max(2, deck.np // 100), differ
    errs = {f: relerr(got[f], orc.get(f)) for f in STATE}
    bad = {f: e for f, e in errs.items() if e > tol}
    assert not bad, errs
    sig = got["sigma"]
    assert np.max(np.abs(sig[:, 0, 1] - sig[:, 1, 0])) > 0.0
    sol.close()
