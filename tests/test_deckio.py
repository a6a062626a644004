"""Deck reader/writer and output writers (CPU only; the oracle drives the
simulations whose output is written)."""
import os

import numpy as np
import pytest

from mcmtop_b200 import deck as D
from mcmtop_b200.deckio import DeckError, deck_text, read_deck
from mcmtop_b200.fortio import fmt_e, fmt_f, fmt_i, read_real, read_record, real_field
from mcmtop_b200.output import Outputs, read_vtk, status_line, vtk_text


# ------------------------------------------------------------ Fortran fields
@pytest.mark.parametrize("field,d,value", [
    ("", 0, 0.0), ("     ", 0, 0.0), ("1.5", 0, 1.5), ("  -2.5e3", 0, -2500.0), ("1.5d-2", 0, 0.015),
    ("1.5+3", 0, 1500.0), ("1.5-3", 0, 0.0015), ("12345", 5, 0.12345), ("12345", 0, 12345.0),
    ("1 2.5", 0, 12.5), (".5", 0, 0.5), ("-.5E1", 0, -5.0), ("3e2", 2, 3.0), ("+7.", 0, 7.0),
])
def test_read_real_fields(field, d, value):
    assert read_real(field, d) == value


def test_read_record_columns():
    # (2i5,e10.0,2i5,e10.0,i5,2e10.0): the material card, format 250 of MCM/mcm_matin.f90:224
    rec = "    2   10      8.93   41                   0       1.5      0.06"
    assert read_record(rec, "(2i5,e10.0,2i5,e10.0,i5,2e10.0)") == [2, 10, 8.93, 41, 0, 0.0, 0, 1.5, 0.06]
    # beyond column 80 nothing is read; short records read blanks
    assert read_record("1" * 79 + "23", "(i80)")[0] == int("1" * 79 + "2")
    assert read_record("    7", "(3i5)") == [7, 0, 0]
    with pytest.raises(ValueError):
        read_record("  1.5", "(i5)")


def test_fortran_output_edit_descriptors():
    assert fmt_e(1234.5, 14, 6) == "  0.123450E+04"
    assert fmt_e(-1.5e-7, 14, 6) == " -0.150000E-06"
    assert fmt_e(0.0, 24, 5) == " " * 13 + "0.00000E+00"
    assert fmt_e(1e-120, 14, 6) == "  0.100000-119"
    assert fmt_e(-0.9999996, 14, 6) == " -0.100000E+01"
    assert fmt_e(12.5, 10, 4) == "0.1250E+02"
    assert fmt_f(-0.5, 15, 8) == "    -0.50000000"
    assert fmt_f(3.24, 15, 8) == "     3.24000000"
    assert fmt_f(1.0e7, 15, 8) == "*" * 15
    assert fmt_i(123456, 5) == "*****" and fmt_i(-12, 5) == "  -12"


def test_real_field_round_trip_is_idempotent():
    rng = np.random.default_rng(7)
    vals = np.concatenate([rng.standard_normal(3000) * 10.0 ** rng.integers(-30, 30, 3000),
                           rng.uniform(-1, 1, 3000), np.round(rng.uniform(-1e7, 1e7, 500))])
    for w, tol in ((10, 5e-3), (20, 1e-12)):
        for v in vals:
            t = real_field(v, w)
            assert len(t) == w and t[0] == " " and "." in t
            back = read_real(t)
            assert abs(back - v) <= tol * abs(v)
            assert real_field(back, w) == t


# ------------------------------------------------------------ deck round trip
def _same_deck(a, b, exact=True):
    tol = 0.0 if exact else 1e-6
    assert a.np == b.np and a.ndim == b.ndim and a.disctype == b.disctype
    np.testing.assert_allclose(b.x, a.x, rtol=0, atol=1e-14 * max(1.0, np.abs(a.x).max()))
    np.testing.assert_allclose(b.v, a.v, rtol=tol, atol=0)
    assert np.array_equal(a.mat, b.mat) and np.array_equal(a.dispbc, b.dispbc)
    assert tuple(a.sym_flag) == tuple(b.sym_flag) and np.allclose(a.sym_x, b.sym_x, rtol=tol)
    assert tuple(a.nthp) == tuple(b.nthp) and np.allclose(a.base_a, b.base_a, rtol=tol)
    for ma, mb in zip(a.materials, b.materials):
        assert (ma.model, ma.eos) == (mb.model, mb.eos)
        for f in ("rho", "mass", "h", "av_l", "av_q"):
            assert abs(getattr(ma, f) - getattr(mb, f)) <= 1e-6 * abs(getattr(ma, f))
        np.testing.assert_allclose(mb.strinput, ma.strinput, rtol=1e-6)
        np.testing.assert_allclose(mb.eosinput, ma.eosinput, rtol=1e-6)


@pytest.mark.parametrize("make", [
    lambda: D.taylor_bar(dx=0.8e-3),
    lambda: D.fluid_column(dx=40e-3),
    lambda: D.taylor_bar(dx=0.8e-3, material=D.sand_model4(1.04), units=D.MMMSG),
], ids=["taylor_model10_eos41", "fluid_model9_eos1", "sand_cap_model4"])
def test_synthetic_decks_round_trip(make):
    d = make()
    text = deck_text(d)
    r = read_deck(text)
    _same_deck(d, r, exact=False)
    assert deck_text(r) == text                       # written, read, written: same text
    assert deck_text(r, comments=False) == "\n".join(
        ln for ln in text.splitlines() if not ln.startswith("$")) + "\n"


HAND_DECK = """\
$ a deck written by hand: comments, two materials out of order, generation cards
Hand deck                                                                      2
*    axopt disctype nummat np
    3    0         2         6         0         0         0
    2.5e-3       0.3       0.0       0.0
    1.0e-4    4    2.0e-4         2    1         0    0    0
    0    1    1    1    0
    0    1    0    1    0    0    0    1
    0    1   60
    0
    2    9     1.000    1    0       0.0    0       0.0       0.0
       0.0       0.1       0.0       0.0
water
    -1.e-5       0.0
       0.0       0.0
       0.0       0.0
       0.0       0.0
       0.0       0.0
       0.0       0.0
eos 1: c1 on the first card, the ninth value alone on the second
       0.0      0.16       0.0       0.0       0.0       0.0       0.0       0.0
       1.0
    1   10      8.93   41    0       0.0    0       1.5      0.06
       0.0      0.05       0.0       0.0
copper
      0.46     0.004     0.001       0.0       0.0       0.0       0.0       0.0
       0.0       0.0       0.0       0.0       0.0       0.0       0.0       0.0
       0.0       0.0       0.0       0.0       0.0       0.0       0.0       0.0
       0.0       0.0       0.0       0.0       0.0       0.0       0.0       0.0
       0.0       0.0       0.0       0.0       0.0       0.0       0.0       0.0
       0.0       0.0       0.0       0.0       0.0       0.0       0.0       0.0
mie-grueneisen
     0.394      1.49       0.0       0.0      2.02       1.0       0.0       0.0
       1    0                 0.0                 0.0                0.05      1
       2    0                0.04                 0.0                0.05      1
       3    7                 0.0                0.04                0.05      1
       4    0                0.04                0.04                0.05      2
       5    0                 0.0                 0.0                0.09      2
       6    0                0.04                 0.0                0.09      2
       1               0.001                0.05                8.93         0.0
       2               0.001                0.05                8.93         0.0
       3               0.001                0.05                8.93         0.0
       4               0.001                0.05                  1.         0.5
       5               0.001                0.05                  1.         0.5
       6               0.001                0.05                  1.         0.5
       2       5
      0.02      0.02      0.07    2
       1       0.0       0.0    -0.019
       3       0.0       0.0    -0.019
       4       0.0       0.0       0.0
       6       0.0       0.0       0.0
         0         0         0         0         1         0
       0.0       0.0       0.0       0.0      0.04       0.0
                 0.0                 0.0              -1.e-9
"""


def test_hand_written_deck():
    d = read_deck(HAND_DECK)
    assert d.title == "Hand deck" and d.np == 6 and len(d.materials) == 2
    m1, m2 = d.materials
    assert (m1.model, m1.eos, m1.rho, m1.av_q, m1.av_l, m1.head) == (10, 41, 8.93, 1.5, 0.06, "copper")
    assert (m2.model, m2.eos, m2.h, m2.head) == (9, 1, 0.1, "water")
    assert m2.strinput[0] == -1e-5 and m2.eosinput[1] == 0.16 and m2.eosinput[8] == 1.0
    assert m1.eosinput[:6].tolist() == [0.394, 1.49, 0.0, 0.0, 2.02, 1.0]
    assert d.endtime == 2.5e-3 and d.tssf == 0.3 and d.state_opt == 4 and d.stpltime == 1e-4
    assert (d.massopt, d.init_h_opt, d.init_rhoe, d.maxnbr) == (1, 1, 0, 60)
    assert d.dispbc.tolist() == [0, 0, 7, 0, 0, 0] and d.mat.tolist() == [1, 1, 1, 2, 2, 2]
    assert d.pardata[3].tolist() == [1e-3, 0.05, 1.0, 0.5]
    assert d.thnodes == (2, 5) and d.transducers == (((0.02, 0.02, 0.07), 2),)
    # generation: node 1 and 3 cards fill 1..3; 4 and 6 fill 4..6
    assert d.v[:, 2].tolist() == [-0.019] * 3 + [0.0] * 3
    assert d.sym_flag == (0, 0, 0, 0, 1, 0) and d.sym_x[4] == 0.04
    assert d.nthp == (0, 0, 1) and d.base_a == (0.0, 0.0, -1e-9)
    again = read_deck(deck_text(d))
    _same_deck(d, again)
    assert deck_text(again) == deck_text(d)


V1_DECK = """\
Version one                                                                    1
    3    5         1         2         0         0
       1.0       0.0
       0.0       0.0         0    0    0
         1    0   30
    0    0    1    0    0    1
    1    9       1.0    1    0       0.0    0       0.0       0.0
       2.0       0.1       0.0       0.0
fluid
       0.0       0.0
       0.0       0.0
       0.0       0.0
       0.0       0.0
       0.0       0.0
       0.0       0.0
eos
       0.0       1.0       0.0       0.0       0.0       0.0       0.0       0.0
       1.0
       1    0                 0.0                 0.0                 0.1      1
       2    0                 0.1                 0.0                 0.1      1
       1       0.1       0.0       0.0
       2       0.1       0.0       0.0
       0.0       1.0       0.0       1.0       0.0       1.0
    1    1    0    1    0    1
"""


def test_version_one_deck():
    # MCM/mcm_read_cont_v1.f90: disctype 5 is read as 1; MCM/mcm_inp_symmetry_v1.f90:
    # coordinates first, and a zero flag makes the plane a symmetry plane
    d = read_deck(V1_DECK)
    assert d.disctype == 1 and d.init_v_opt == 1 and d.tcrit_opt == 1 and d.mirr_opt == 1
    assert d.sym_flag == (0, 0, 1, 0, 1, 0) and d.sym_x == (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    assert d.v[:, 0].tolist() == [0.1, 0.1] and d.status_interval == 100


def _mutate(old, new, count=1):
    assert old in HAND_DECK
    return HAND_DECK.replace(old, new, count)


@pytest.mark.parametrize("text,match", [
    (_mutate("Hand deck                                                                      2",
             "Hand deck                                                                      3"), "version 3"),
    (_mutate("       2    0                0.04", "       5    0                0.04"), "out of order"),
    (_mutate("0.05      1\n       4", "0.05      0\n       4"), "zero material"),
    (_mutate("0.05      1\n       4", "0.05      3\n       4"), "beyond"),
    (_mutate("    2    9     1.000    1", "    2    3     1.000    1"), "not permitted"),
    (_mutate("    1   10      8.93   41", "    1   10      8.93    0"), "requires an equation"),
    (_mutate("    1   10      8.93   41", "    1   10      8.93   42"), "eos type"),
    (_mutate("    1   10      8.93   41", "    3   10      8.93   41"), "out of range"),
    (_mutate("    2    9     1.000    1", "    1    9     1.000    1"), "no material 2"),
    (_mutate("       3       0.0       0.0    -0.019", "       3       0.0       0.0    -0.018"), "not constant"),
    (_mutate("       1       0.0       0.0    -0.019", "       2       0.0       0.0    -0.019"), "not for node 1"),
    (_mutate("       4       0.0       0.0       0.0\n       6",
             "       2       0.0       0.0       0.0\n       6"), "less than previous"),
    (_mutate("         0         0         0         0         1         0",
             "         2         0         0         0         1         0"), "periodic"),
    (_mutate("    3    0         2", "    4    0         2"), "axisymmetry"),
    (_mutate("    2.5e-3       0.3", "    2.5x-3       0.3"), "2nd control card"),
    (HAND_DECK[:HAND_DECK.index("      0.02      0.02")], "end of file"),
], ids=lambda p: p if isinstance(p, str) and len(p) < 40 else "")
def test_deck_errors(text, match):
    with pytest.raises(DeckError, match=match):
        read_deck(text)


def test_more_than_ten_history_particles():
    # MCM/mcm_nodehist.f90:43 stores item l of card i at i+l: with 11 ids the
    # 11th position is never set, which the reader reports
    d = read_deck(HAND_DECK)
    with pytest.raises(ValueError, match="at most 10"):
        deck_text(d.replace(thnodes=tuple(range(1, 12))))
    lines = HAND_DECK.replace("    2.0e-4         2    1", "    2.0e-4        11    1").splitlines()
    k = lines.index("       2       5")
    lines[k:k + 1] = ["".join(f"{i:8d}" for i in range(1, 11)), "       1"]
    with pytest.raises(DeckError, match="at most 10"):
        read_deck("\n".join(lines) + "\n")


# ----------------------------------------------------- simulations from decks
def _grid_bar(nx=6, nz=10, dx=0.04):
    """A bar of exactly representable lattice coordinates, so that the deck
    holds the same doubles as the generator."""
    g = (np.arange(nx) - nx / 2 + 0.5) * dx
    z = (np.arange(nz) + 0.5) * dx
    Z, Y, X = np.meshgrid(z, g, g, indexing="ij")
    x = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    base = D.taylor_bar(dx=0.8e-3)
    mat = D.copper_model10(0.052)
    mat.mass = round(mat.rho * x.shape[0] * dx ** 3, 9)
    mat.strinput[0] = 0.46          # 46e9 * 1e-11 is not the double nearest 0.46
    v = np.zeros_like(x)
    v[:, 2] = -0.019
    return base.replace(x=x, v=v, materials=[mat], mat=np.ones(len(x), np.int32),
                        dispbc=np.zeros(len(x), np.int32), name="grid_bar", title="grid bar")


def test_deck_text_drives_the_same_simulation(oracle_lib):
    from oracle.pyoracle import Oracle

    d = _grid_bar()
    text = deck_text(d)
    r = read_deck(text)
    assert np.array_equal(r.x, d.x) and r.materials[0].mass == d.materials[0].mass
    a, b = Oracle(d), Oracle(r)
    try:
        for _ in range(8):
            a.step()
            b.step()
        for f in ("x", "v", "sigma", "rho", "e", "p"):
            assert np.array_equal(a.get(f), b.get(f)), f
    finally:
        a.close()
        b.close()


def oracle_state(orc, fields):
    out = {}
    for f in fields:
        out[f] = orc.get_int(f) if f in ("mat", "ptype", "nnbr") else orc.get(f)
    return out


def oracle_program(deck, base, directory, steps):
    """The loop of mcmtop_b200.run.Program driven by the oracle (no fusing)."""
    from oracle.pyoracle import Oracle

    class Recording(Outputs):
        def state_output(self, state):
            self.last_state = state
            super().state_output(state)

        def timehist(self, ptime, state, energies, contact_forces=None):
            self.last_th = (ptime, state, energies.copy())
            super().timehist(ptime, state, energies, contact_forces)

    orc = Oracle(deck)
    out = Recording(deck, base, directory)
    need = out.fields(True, True)
    out.initial(orc.scalar("ptime"), oracle_state(orc, need), orc.energies())
    for _ in range(steps):
        orc.step_a()
        orc.dt_update()
        orc.step_b()
        t = orc.scalar("ptime")
        st, th = out.due(t)
        if st or th:
            cf = orc.contact_forces() if (th and deck.contacttype > 0) else None
            out.after_energies(t, oracle_state(orc, out.fields(st, th)), orc.energies(), cf)
        if orc.ended():
            break
        orc.step_c()
    return orc, out


def test_outputs_follow_the_state(tmp_path, oracle_lib):
    d = _grid_bar().replace(state_opt=4, stpltime=0.1, thpltime=0.0, thnodes=(1, 17, 200),
                            transducers=(((0.0, 0.0, 0.2), 1),), status_interval=5)
    orc, out = oracle_program(d, "bar", str(tmp_path), 12)
    try:
        names = sorted(os.listdir(tmp_path))
        assert "bar0.vtk" in names and "1bar0.vtk" in names and "2bar0.vtk" in names
        assert {"bar_thist.csv", "bar_th1.csv", "bar_th17.csv", "bar_th200.csv", "bar_ptrn.csv",
                "bar_vtrn.csv"} <= set(names)
        last = max(int(n[3:-4]) for n in names if n.startswith("bar") and n.endswith(".vtk"))
        assert last == out.istate - 1 >= 1
        # the newest state file holds the state of its output step (F15.8, E24.5)
        st = out.last_state
        vt = read_vtk(str(tmp_path / f"bar{last}.vtk"))
        np.testing.assert_allclose(vt["x"], st["x"], rtol=0, atol=5.1e-9)
        np.testing.assert_allclose(vt["v"], st["v"], rtol=0, atol=5.1e-9)
        np.testing.assert_allclose(vt["Stress_Z"], st["sigma"][:, 2, 2], rtol=5e-5, atol=1e-300)
        np.testing.assert_allclose(vt["Pressure"], st["p"], rtol=5e-5, atol=1e-300)
        m1 = read_vtk(str(tmp_path / f"1bar{last}.vtk"))
        assert m1["x"].shape == vt["x"].shape and "PTYPE" in m1
        m2 = read_vtk(str(tmp_path / f"2bar{last}.vtk"))
        assert m2["x"].shape == (0, 3)
        # one time-history row per step plus the initial one
        rows = (tmp_path / "bar_th17.csv").read_text().splitlines()
        assert rows[1] == "Time history data for particle     17"
        assert len(rows) == 3 + 13
        vals = [float(s) for s in rows[-1].split(",")[1:-1]]
        assert len(vals) == 20
        ptime, th, energies = out.last_th
        # e14.6 keeps 6 significant digits
        assert abs(vals[0] - ptime) <= 5e-6 * ptime
        np.testing.assert_allclose(vals[1:4], th["x"][16], rtol=5e-6)
        np.testing.assert_allclose(vals[7], th["rho"][16], rtol=5e-6)
        np.testing.assert_allclose(vals[16], th["e"][16] / th["mass"][16], rtol=5e-6)
        glob = (tmp_path / "bar_thist.csv").read_text().splitlines()
        assert glob[1] == "Global time history data" and len(glob) == 2 + 13
        ke = float(glob[-1].split(",")[2])
        assert abs(ke - energies[0]) <= 5e-6 * abs(ke)
        ptrn = (tmp_path / "bar_ptrn.csv").read_text().splitlines()
        assert float(ptrn[-1].split(",")[1]) != 0.0
    finally:
        orc.close()


def test_vtk_record_layout():
    st = {"x": np.array([[0.5, -0.25, 1.0], [1e-9, 2.0, 3.5]]), "v": np.array([[0.0, 0.0, -0.019], [1.0, 2.0, 3.0]]),
          "p": np.array([1.5e-3, -2.0]), "sigma": np.zeros((2, 3, 3)), "mat": np.array([1, 2], np.int32),
          "ptype": np.array([0, 3], np.int32)}
    st["sigma"][0] = [[1.0, 0.5, 0.0], [0.5, 2.0, 0.0], [0.0, 0.0, 3.0]]
    t = vtk_text(st).splitlines()
    assert t[:5] == ["# vtk DataFile Version 3.0", "TEST", "ASCII", "DATASET UNSTRUCTURED_GRID",
                     " POINTS 2                         double"]
    assert t[5] == "     0.50000000    -0.25000000     1.00000000"
    assert t[6] == "     0.00000000     2.00000000     3.50000000"
    assert t[7] == " CELLS 2                         4                        "
    assert t[8:10] == ["1      0", "1      1"]
    assert t[10:13] == ["CELL_TYPES     2", "1", "1"]
    assert t[13:15] == ["POINT_DATA     2", " VECTORS Velocities double"]
    assert t[17:21] == ["SCALARS Pressure double 1", "LOOKUP_TABLE default",
                        "             0.15000E-02", "            -0.20000E+01"]
    # von Mises of (1, 2, 3; 0.5): sqrt(0.5 (1 + 1 + 4 + 6 * 0.25)) = sqrt(3.75)
    k = t.index("SCALARS VM_Stress double 1")
    assert t[k + 2] == fmt_e(float(np.float32(np.sqrt(3.75))), 24, 5)
    m = vtk_text(st, np.array([1]), with_ptype=True).splitlines()
    assert m[-3:] == ["SCALARS PTYPE double 1", "LOOKUP_TABLE default", "    3"]
    assert status_line(100, 1.5e-5, 2.5e-8).splitlines()[1:] == [
        "     Problem status for time-step    100", "     Time: 0.1500E-04     dt: 0.2500E-07"]


def test_relaxed_state_layout():
    from mcmtop_b200.output import drelax_text
    st = {"x": np.array([[0.5, -1.25e-3, 3.0]]), "dispbc": np.array([7]), "mat": np.array([2]),
          "mass": np.array([1e-3]), "h": np.array([0.052]), "rho": np.array([8.93]), "e": np.array([12.5])}
    t = drelax_text(st).splitlines()
    assert t[:3] == ["*", "* Node Coordinates and Materials", "*"]
    assert t[3] == "       1    7 0.5000000000000E+00-0.1250000000000E-02 0.3000000000000E+01      2"
    assert len(t[3]) == 80
    assert t[7] == "       1 0.1000000000000E-02 0.5200000000000E-01 0.8930000000000E+01 0.1250000000000E+02"
    # the node card reads back with the deck's node format; the data card is
    # 88 columns wide, and an 80-column reader loses the energy's exponent
    assert read_record(t[3], "(i8,i5,3e20.0,i7)") == [1, 7, 0.5, -1.25e-3, 3.0, 2]
    assert read_record(t[7], "(i8,4e20.0)")[4] == 0.125


def test_ensight_records():
    from mcmtop_b200.output import _ens_scalar, _ens_vector, ensight_geometry_text, ensight_res_text
    # six scalars per record, the rest on the last one; |v| < 1e-50 written as zero
    assert _ens_scalar(np.array([1.0, -2.0, 3.0, 4.0, 5.0, 6.0, 1e-60])) == [
        " 0.10000E+01-0.20000E+01 0.30000E+01 0.40000E+01 0.50000E+01 0.60000E+01\n", " 0.00000E+00\n"]
    # vectors: two particles per record, in groups of six particles
    v = np.arange(21, dtype=float).reshape(7, 3)
    rec = _ens_vector(v)
    assert len(rec) == 4 and rec[3] == " 0.18000E+02 0.19000E+02 0.20000E+02\n"
    g = ensight_geometry_text(np.array([[0.5, -0.25, 1.0], [1.0, 2.0, 3.0]]), np.array([1, 1]), 1).splitlines()
    assert g[:5] == [" frame geometry", " node id assign", " element id assign", " coordinates", "      2"]
    assert g[5] == " 0.50000E+00-0.25000E+00 0.10000E+01"
    assert g[7:] == ["part 1", "points list of part 1", " point", "       2", "       1", "       2"]
    # the results file lists the times before the state just written
    r = ensight_res_text("bar", 3, ["  0.000000E+00", "  0.123456E+01", "  0.250000E+01"]).splitlines()
    assert r[:4] == [" 18 3 0", "  2", " 0.000E+00 0.123E+01", " 1 1"]
    assert r[4] == " bar_density*** density" and r[-1] == " bar_accelera*** acceleration" and len(r) == 25


def test_ensight_outputs_follow_the_state(tmp_path, oracle_lib):
    d = _grid_bar().replace(state_opt=1, stpltime=0.1, thpltime=1e9)
    orc, out = oracle_program(d, "bar", str(tmp_path), 8)
    try:
        names = set(os.listdir(tmp_path))
        assert {"bar.geo", "bar.res", "bar_time.txt", "bar_density001", "bar_displace001", "bar_material001"} <= names
        last = out.istate - 1
        assert last >= 2 and f"bar_sigma23{last:03d}" in names
        st = out.last_state
        def fields12(path):     # e12.5 fields, which touch when a value is negative
            lines = path.read_text().splitlines()
            return lines[0], np.array([float(ln[k:k + 12]) for ln in lines[1:] for k in range(0, len(ln), 12)])

        head, dens = fields12(tmp_path / f"bar_density{last:03d}")
        assert head == " density" and len(dens) == d.np
        np.testing.assert_allclose(dens, st["rho"], rtol=5e-5)
        _, disp = fields12(tmp_path / f"bar_displace{last:03d}")
        np.testing.assert_allclose(disp.reshape(-1, 3), st["x"] - d.x, rtol=5e-5, atol=1e-9)
        times = (tmp_path / "bar_time.txt").read_text().splitlines()
        assert len(times) == last
        res = (tmp_path / "bar.res").read_text().splitlines()
        assert int(res[1]) == last - 1
    finally:
        orc.close()


def test_node_cards_bulk_and_card_by_card_agree():
    # plain numbers are read in bulk; a card with a D exponent or a blank
    # field sends the block through the card-by-card Fortran rules
    d = _grid_bar()
    text = deck_text(d)
    plain = read_deck(text)
    lines = text.splitlines()
    k = next(i for i, ln in enumerate(lines) if ln.startswith("       7    0"))
    rec = lines[k]
    lines[k] = rec[:8] + "     " + f"{'-1.25d-1':>20}" + rec[33:]
    odd = read_deck("\n".join(lines) + "\n")
    assert odd.x[6, 0] == -0.125 and odd.dispbc[6] == 0
    same = np.ones(d.np, bool)
    same[6] = False
    assert np.array_equal(odd.x[same], plain.x[same]) and np.array_equal(odd.x[6, 1:], plain.x[6, 1:])
    assert np.array_equal(odd.mat, plain.mat)
