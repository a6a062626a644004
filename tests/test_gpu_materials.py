"""Parity of the other material models and equations of state with the oracle.

The Taylor bar and the fluid column exercise model 10 + EOS 41 and model 9 +
EOS 1.  The cases below run the remaining ported families through the same
step: the isotropic elastic model 1 (MCM/mcm_f3dm1.f90), the kinematic/
isotropic hardening model 3 (MCM/mcm_f3dm3.f90), and the polynomial (1),
DYNA Grueneisen (4), ideal gas (13) and Tait (28) equations of state
(MCM/mcm_eos*c.f90, MCM/mcm_eqos*.f90) under model 10 or the null model 9.
Card values are in the cm-g-us system of the decks.  The CPU test checks
that the oracle itself runs every case to finite fields; the GPU tests
compare the FP64-exact step with it after a few steps and the fast FP64 step
at the looser tolerance of the other parity tests.
"""
import dataclasses

import numpy as np
import pytest

from mcmtop_b200 import _abi
from mcmtop_b200.deck import MaterialCard, copper_model10, fluid_column, taylor_bar, water_model9
from mcmtop_b200.solver import Solver
from oracle.pyoracle import Oracle

STATE = ["x", "v", "rho", "e", "p", "c", "efps", "sigma", "q"]
NSTEPS = 12
DX_BAR = 0.8e-3
RHO_CU = 8.93
C0_CU = 0.394            # cm/us


def _solid(model):
    """Models 1 and 3 (no EOS).  The cards fill the first row of the 5-row
    constant table cm(i, j) = strinput(i + 5(j-1)): Young's modulus cm(1,1),
    Poisson ratio cm(1,2), yield stress cm(1,3), tangent modulus cm(1,4),
    hardening parameter beta cm(1,5) (MCM/mcm_sets1.f90:23-51,
    MCM/mcm_sets3.f90:23-43, MCM/mcm_f3dm3.f90)."""
    card = MaterialCard(model=model, eos=0, rho=RHO_CU, av_l=0.06, av_q=1.5)
    card.strinput[0] = 1.2
    card.strinput[5] = 0.34
    card.strinput[10] = 4.0e-3
    card.strinput[15] = 1.0e-2
    card.strinput[20] = 0.5
    return card


def _model10_eos(eos):
    card = copper_model10(0.0)
    card.eos = eos
    card.eosinput[:] = 0.0
    if eos == 1:          # linear polynomial: c1 = rho0 c0^2; relative volume 1
        card.eosinput[1] = RHO_CU * C0_CU ** 2
        card.eosinput[8] = 1.0
    elif eos == 4:        # c, s1, s2, s3, gamma0, a, e0, v0 (MCM/mcm_eos4c.f90)
        card.eosinput[:8] = [C0_CU, 1.49, 0.0, 0.0, 2.02, 0.47, 0.0, 1.0]
    elif eos == 28:       # Tait: B, gamma, e0, v0
        card.eosinput[:4] = [RHO_CU * C0_CU ** 2 / 4.0, 4.0, 0.0, 1.0]
    return card


def _gas():
    """Null material with the ideal-gas EOS 13: gamma, -, e0 (per unit
    volume), v0; strinput(1) is the pressure floor."""
    card = MaterialCard(model=9, eos=13, rho=1.2e-3, av_l=0.06, av_q=1.5)
    card.strinput[0] = 0.0
    card.eosinput[:4] = [1.4, 0.0, 2.5e-6, 1.0]
    return card


def _tait_water():
    card = water_model9(0.0)
    card.eos = 28
    card.eosinput[:] = 0.0
    card.eosinput[:4] = [card.rho * (40.0e-4) ** 2 / 7.0, 7.0, 0.0, 1.0]
    return card


def _bar(card, velocity=190.0):
    return taylor_bar(dx=DX_BAR, velocity=velocity, material=card)


def _column(card):
    d = fluid_column(dx=0.01, block=(0.1, 0.06, 0.2), box=(0.4, 0.06, 0.3))
    m = d.materials[0]
    card = dataclasses.replace(card, h=m.h, mass=card.rho * d.np * (0.01 * 100) ** 3)
    return d.replace(materials=[card])


CASES = {
    "model1_elastic": lambda: _bar(_solid(1), velocity=50.0),
    "model3_kinematic": lambda: _bar(_solid(3)),
    "model10_eos1": lambda: _bar(_model10_eos(1)),
    "model10_eos4": lambda: _bar(_model10_eos(4)),
    "model10_eos28": lambda: _bar(_model10_eos(28)),
    "model9_eos13_gas": lambda: _column(_gas()),
    "model9_eos28_water": lambda: _column(_tait_water()),
}


def relerr(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = float(np.max(np.abs(b))) if b.size else 0.0
    if scale == 0.0:
        return float(np.max(np.abs(a))) if a.size else 0.0
    return float(np.max(np.abs(a - b)) / scale)


@pytest.mark.parametrize("case", sorted(CASES))
def test_oracle_runs_case(case):
    deck = CASES[case]()
    orc = Oracle(deck)
    for _ in range(NSTEPS):
        orc.step()
    for f in STATE:
        assert np.all(np.isfinite(orc.get(f))), (case, f)
    assert np.max(np.abs(orc.get("sigma"))) > 0.0 or case.startswith("model9")


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_material_parity_exact(gpu_lib, case):
    deck = CASES[case]()
    sol = Solver(deck, _abi.PREC_FP64_EXACT)
    orc = Oracle(deck)
    for _ in range(NSTEPS):
        sol.step()
        orc.step()
    got = sol.download(STATE)
    bad = {f: relerr(got[f], orc.get(f)) for f in STATE}
    bad = {f: e for f, e in bad.items() if e > 1e-10}
    assert not bad, (case, bad)
    assert abs(sol.ptime - orc.scalar("ptime")) <= 1e-12 * orc.scalar("ptime")
    sol.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_material_parity_fast(gpu_lib, case):
    deck = CASES[case]()
    sol = Solver(deck, _abi.PREC_FP64)
    orc = Oracle(deck)
    for _ in range(NSTEPS):
        sol.step()
        orc.step()
    got = sol.download(STATE)
    bad = {f: relerr(got[f], orc.get(f)) for f in STATE}
    bad = {f: e for f, e in bad.items() if e > 1e-9}
    assert not bad, (case, bad)
    sol.close()
