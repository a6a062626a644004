"""CPU checks of the C-ABI library: it loads, exports every entry point that
include/mcm_gpu.h declares, its structures match the ctypes mirror, and its
host-side deck processing agrees with the oracle.  No device calls."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

from mcmtop_b200 import _abi
from mcmtop_b200.deck import fluid_column, taylor_bar, MaterialCard

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(_abi.LIB_PATH):
        from mcmtop_b200 import build

        build.build()
    return _abi.load()


def test_exports_every_declared_symbol(lib):
    names = _abi.exported_symbols()
    assert len(names) >= 18
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        assert hasattr(lib, n)


def test_abi_version_and_strerror(lib):
    assert lib.mcm_gpu_abi_version() == 3
    assert lib.mcm_gpu_strerror(_abi.MCM_ENBR_OVERFLOW) == b"neighbour table overflow"
    assert lib.mcm_gpu_strerror(12345) == b"unknown status"


def test_struct_layout_matches_header():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "mcm_gpu.h"
int main(void) {
  printf("%zu %zu %zu %zu\n", sizeof(mcm_gpu_material), sizeof(mcm_gpu_config), sizeof(mcm_gpu_fields), sizeof(mcm_gpu_time));
  printf("%zu %zu %zu %zu\n", offsetof(mcm_gpu_material, strinput), offsetof(mcm_gpu_config, boundary_x),
         offsetof(mcm_gpu_config, precision), offsetof(mcm_gpu_fields, mat));
  printf("%zu %zu %zu\n", sizeof(mcm_gpu_tuning), offsetof(mcm_gpu_tuning, adj_kind), offsetof(mcm_gpu_tuning, ms_per_step));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        with open(c, "w") as fh:
            fh.write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        lines = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    sizes = [int(t) for t in lines[0].split()]
    offs = [int(t) for t in lines[1].split()]
    assert sizes == [C.sizeof(_abi.Material), C.sizeof(_abi.Config), C.sizeof(_abi.Fields), C.sizeof(_abi.Time)]
    assert offs == [_abi.Material.strinput.offset, _abi.Config.boundary_x.offset, _abi.Config.precision.offset,
                    _abi.Fields.mat.offset]
    tun = [int(t) for t in lines[2].split()]
    assert tun == [C.sizeof(_abi.Tuning), _abi.Tuning.adj_kind.offset, _abi.Tuning.ms_per_step.offset]


def _lib_material(lib, card):
    m = _abi.Material()
    m.model, m.eos, m.visc_type = card.model, card.eos, card.visc_type
    m.rho, m.av_l, m.av_q, m.mass, m.h = card.rho, card.av_l, card.av_q, card.mass, card.h
    for i in range(48):
        m.strinput[i] = float(card.strinput[i])
    for i in range(24):
        m.eosinput[i] = float(card.eosinput[i])
    st = lib.mcm_gpu_material_from_deck(C.byref(m))
    return st, m


@pytest.mark.parametrize("which", ["model10", "model9", "model1", "model3"])
def test_material_processing_matches_oracle(lib, which):
    from oracle.pyoracle import Oracle

    deck = taylor_bar(dx=1.6e-3)
    if which == "model9":
        deck = fluid_column(dx=0.02, block=(0.1, 0.06, 0.1), box=(0.2, 0.06, 0.2))
    elif which in ("model1", "model3"):
        card = MaterialCard(model=int(which[-1]), eos=0, rho=8.93, h=deck.materials[0].h)
        card.strinput[0] = 1.2          # Young's modulus (Mbar)
        card.strinput[1] = 0.34         # Poisson ratio
        card.strinput[2] = 4e-3         # yield
        card.strinput[3] = 1e-2         # tangent modulus
        card.strinput[4] = 0.5          # beta
        card.mass = deck.materials[0].mass
        deck = deck.replace(materials=[card])
    st, m = _lib_material(lib, deck.materials[0])
    assert st == 0
    orc = Oracle(deck)
    si, ei, g = orc.material_table(1)
    assert np.array_equal(np.array(m.strinput[:]), si)
    assert np.array_equal(np.array(m.eosinput[:]), ei)
    assert m.g == g


def test_material_rejects_eos_on_solid(lib):
    card = MaterialCard(model=1, eos=41, rho=8.93)
    st, _ = _lib_material(lib, card)
    assert st == _abi.MCM_EINVAL


def test_cap_model_card_without_soil_type_is_rejected(lib):
    """Model 4 is set up by the library (mcm_sets4); a card whose ltype is
    neither soil (1) nor rock (2) has no mode in the cap model's table."""
    card = MaterialCard(model=4, eos=0, rho=2.0)
    st, _ = _lib_material(lib, card)
    assert st == _abi.MCM_EINVAL
