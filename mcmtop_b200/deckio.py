"""MCM input decks (``<name>.mcm``): reader and writer.

The reader restates MCM's input routines card by card, with their formats,
defaults left to the solver set-up, order checks and error conditions:

* MCM/mcm_getinput.f90:37-128      title card ``(a78,i2)``, version dispatch
* MCM/mcm_control_v2.f90:88-124    the seven control cards of version 2
* MCM/mcm_read_cont_v1.f90:40-90   the five control cards of version 1
* MCM/mcm_matin.f90:41-148         material cards, properties, EOS cards
* MCM/mcm_nodein.f90:33-115        node cards and additional particle cards
* MCM/mcm_nodehist.f90:29-62       time-history particle cards
* MCM/mcm_transducers_in.f90:26-41 pressure-transducer cards
* MCM/mcm_Inputvel.f90:32-108      initial velocities with generation
* MCM/mcm_inp_symmetry_v2.f90:29-137, MCM/mcm_inp_symmetry_v1.f90:29-80
                                   boundary planes
* MCM/mcm_contactype.f90:27-47     contact cards
* MCM/mcm_baseaccel_in.f90:23-33   base accelerations
* MCM/mcm_gttxsg.f90:22-31         card reader: lines whose first column is
                                   ``*`` or ``$`` are comments

The writer produces version-2 decks that the reference reads back: every
real field holds the most precise text that fits its width, so a deck
written, read and written again is the same text.  Fields of 10 columns
keep 7 to 9 significant digits, the 20-column coordinate fields 15 to 17.

Deliberate differences from the reference: an error raises DeckError with
the card's line number instead of stopping the program; a node card whose
material number exceeds the number of materials, and a material number that
no material card defines, are errors here (the reference indexes out of its
arrays); more than 10 time-history particles are an error (see
read_thnodes).
"""
from __future__ import annotations

import io
import os

import numpy as np

from .deck import Deck, MaterialCard
from .fortio import FieldError, int_field, read_record, real_field

# MCM/mcm_matin.f90:72-148: property and EOS card layouts
_PROP_CARDS = {1: (6, 5), 3: (6, 5), 4: (6, 5), 9: (6, 5), 10: (6, 8)}
_EOS_CARDS = {1: ((8, "(8e10.0)"), (1, "(8e10.0)")), 4: ((8, "(8e10.0)"),), 13: ((5, "(5e10.0)"),),
              28: ((2, "(5e10.0)"),), 41: ((8, "(8e10.0)"),)}


class DeckError(ValueError):
    """An input error that makes MCM stop (mcm_termin / mcm_shutdown(2))."""

    def __init__(self, msg: str, line: int | None = None, text: str | None = None):
        where = ""
        if line is not None:
            where = f" (line {line}: {text.rstrip()!r})" if text is not None else f" (line {line})"
        super().__init__(msg + where)
        self.line = line


class _Cards:
    """Card stream of MCM/mcm_gttxsg.f90: skips comment lines, keeps line numbers."""

    def __init__(self, text: str):
        self.lines = text.splitlines()
        self.pos = 0
        self.line = 0
        self.text = ""

    def next(self, what: str) -> str:
        while self.pos < len(self.lines):
            t = self.lines[self.pos]
            self.pos += 1
            if t[:1] in ("*", "$"):
                continue
            self.line, self.text = self.pos, t
            return t
        raise DeckError(f"{what}: end of file")

    def read(self, what: str, fmt, count: int | None = None) -> list:
        t = self.next(what)
        try:
            return read_record(t, fmt, count)
        except FieldError as e:
            raise DeckError(f"{what}: {e}", self.line, t) from None

    def fail(self, msg: str):
        raise DeckError(msg, self.line, self.text)

    def block(self, n: int) -> tuple:
        """The next n cards and their line numbers (for a bulk parse)."""
        texts, lines = [], []
        while len(texts) < n and self.pos < len(self.lines):
            t = self.lines[self.pos]
            self.pos += 1
            if t[:1] in ("*", "$"):
                continue
            texts.append(t)
            lines.append(self.pos)
        return texts, lines


def _bulk_columns(texts: list, fmt: str):
    """Columns of many cards of one fixed format, converted by numpy; None when
    any field needs the full Fortran rules (blank or embedded-blank fields,
    D or bare-sign exponents, or what numpy reads that a Fortran READ would
    not), in which case the cards are read one by one."""
    from .fortio import parse_format, RECORD
    spec = parse_format(fmt)
    rec = np.array([t.rstrip("\r\n")[:RECORD].ljust(RECORD) for t in texts])
    cols, pos = [], 0
    try:
        for kind, w, d in spec:
            sub = np.array([r[pos:pos + w] for r in rec.tolist()])
            pos += w
            # numpy also takes forms a Fortran READ does not ("1_0", "nan"): keep to the plain ones
            if (np.char.find(sub, "_") >= 0).any():
                return None
            if kind == "i":
                col = sub.astype(np.int64)
            else:
                if d:
                    return None
                col = sub.astype(np.float64)
                if not np.all(np.isfinite(col)):
                    return None
            cols.append(col)
    except ValueError:
        return None
    return cols


# ------------------------------------------------------------------ reading
def read_deck(source) -> Deck:
    """Reads a deck from a path, a file object or the deck text itself."""
    if hasattr(source, "read"):
        text, name = source.read(), "deck"
    elif isinstance(source, (str, os.PathLike)) and os.path.exists(source):
        with open(source) as f:
            text = f.read()
        name = os.path.splitext(os.path.basename(os.fspath(source)))[0]
    elif isinstance(source, str) and "\n" in source:
        text, name = source, "deck"
    else:
        raise FileNotFoundError(source)
    cards = _Cards(text)
    title, vern = cards.read("error reading title card", "(a78,i2)")
    d = {"title": title.rstrip(), "name": name}
    if vern == 2:
        _control_v2(cards, d)
    elif vern == 1:
        _control_v1(cards, d)
    else:
        cards.fail(f"Input file version {vern} is not supported in this version of the code")
    ndim, np_ = d["ndim"], d["np"]
    d["materials"] = _materials(cards, d["nummat"])
    _nodes(cards, d)
    if d.pop("thnode") > 0:
        d["thnodes"] = read_thnodes(cards, d["_thnode"], np_)
    ntr = d.pop("num_transducer")
    if ntr > 0:
        tr = []
        for _ in range(ntr):
            vals = cards.read("Error in pressure transducer cards", f"({ndim}e10.0,i5)")
            tr.append((tuple(vals[:ndim]) + (0.0,) * (3 - ndim), vals[ndim]))
        d["transducers"] = tuple(tr)
    d["v"] = _velocities(cards, d)
    if d["mirr_opt"] == 1:
        if vern == 2:
            _symmetry_v2(cards, d)
        else:
            _symmetry_v1(cards, d)
    if vern == 2 and d["contacttype"] > 0:
        ncm, opt = cards.read(" error reading contact definitions", "(2i5)")
        d["ncontmats"], d["cont_opt"] = ncm, opt
        if ncm == -1:
            kc, nc = [], []
            for _ in range(d["nummat"]):
                k, n = cards.read(" error reading contact definitions", "(2e10.5)")
                kc.append(k)
                nc.append(n)
            d["k_cont"], d["n_cont"] = tuple(kc), tuple(nc)
    if vern == 2 and any(t == 1 for t in d["nthp"]):
        a = cards.read("Error reading base accelerations card", "(3e20.0)")
        d["base_a"] = tuple(a[k] if d["nthp"][k] == 1 else 0.0 for k in range(3))
    for k in [k for k in d if k.startswith("_")] + ["nummat", "np"]:
        d.pop(k, None)
    return Deck(**d)


def _control_v2(cards: _Cards, d: dict) -> None:
    """MCM/mcm_control_v2.f90:88-124 and the checks of :193-243."""
    v = cards.read(" error reading 1st control card", "(2i5,5i10)")
    axopt, d["disctype"], d["nummat"], d["np"], d["max_np"], d["nstressp"], d["nvelocp"] = v
    v = cards.read(" error reading 2nd control card", "(4e10.0)")
    d["endtime"], d["tssf"], d["itss"], d["drelax_scale"] = v
    v = cards.read(" error reading 3rd control card", "(e10.0,i5,e10.0,i10,i5,i10,2i5)")
    (d["stpltime"], d["state_opt"], d["thpltime"], d["thnode"], d["num_transducer"], d["status_interval"],
     d["restart_interval"], d["run_restart"]) = v
    v = cards.read(" error reading 4th control card", "(5i5)")
    d["keep_files"], d["init_v_opt"], d["massopt"], d["init_h_opt"], d["init_rhoe"] = v
    v = cards.read(" error reading 5th control card", "(10i5)", 8)
    d["contacttype"], d["tcrit_opt"], d["veloc_opt"], d["mirr_opt"], d["nlcur"] = v[:5]
    d["nthp"] = tuple(v[5:8])
    d["h_opt"], d["krtype"], d["maxnbr"] = cards.read(" error reading 6th control card", "(3i5)")
    cards.next(" error reading 7th control card")      # not used in version 2
    _axopt(cards, d, axopt, "2D axisymmetry is not supported in version 2")
    d["_thnode"] = d["thnode"]


def _control_v1(cards: _Cards, d: dict) -> None:
    """MCM/mcm_read_cont_v1.f90:40-90 (defaults :27-37, disctype renumbering :120-133)."""
    v = cards.read(" error reading 1st control card", "(2i5,4i10)")
    axopt, disc, d["nummat"], d["np"], d["nstressp"], d["nvelocp"] = v
    d["endtime"], d["tssf"], d["itss"] = cards.read(" error reading 2nd control card", "(3e10.0)")
    v = cards.read(" error reading 3rd control card", "(2e10.0,i10,i5,i5)")
    d["stpltime"], d["thpltime"], d["thnode"], d["num_transducer"], d["state_opt"] = v
    d["krtype"], d["init_h_opt"], d["maxnbr"] = cards.read(" error reading 4th control card", "(i10,2i5)")
    v = cards.read(" error reading 5th control card", "(7i5)", 6)
    d["contacttype"], d["massopt"], d["tcrit_opt"], d["veloc_opt"], d["h_opt"], d["mirr_opt"] = v
    d["init_v_opt"], d["init_rhoe"], d["status_interval"], d["nthp"] = 1, 0, 100, (0, 0, 0)
    _axopt(cards, d, axopt, "2D axisymmetry is not supported")
    if disc == 5:
        disc = 1
    elif disc == 3:
        disc = 2
    elif disc in (1, 2):
        cards.fail(f"Discretisation type {disc} is not supported in version 1 input")
    d["disctype"] = disc
    d["_thnode"] = d["thnode"]


def _axopt(cards: _Cards, d: dict, axopt: int, msg: str) -> None:
    if axopt == 4:
        cards.fail(msg)
    if axopt not in (1, 2, 3):
        cards.fail(f"axis option {axopt} is not 1, 2 or 3")
    d["ndim"] = axopt


def _materials(cards: _Cards, nummat: int) -> list:
    """MCM/mcm_matin.f90:41-148; card values are kept as read (the defaults
    of :47-57 are applied by the solver's material set-up)."""
    mats = [None] * nummat
    for _ in range(nummat):
        n, model, rho, eos, ihq, qh, vt, avq, avl = cards.read(
            " error reading material control card", "(2i5,e10.0,2i5,e10.0,i5,2e10.0)")
        line = cards.line
        mass, h, rmin, rmax = cards.read(" error reading MCM material options card", "(4e10.0)")
        if n <= 0 or n > nummat:
            raise DeckError("error in input - material number is out of range", line)
        if model in (1, 3, 4):
            if eos != 0:
                raise DeckError(f"material {n}: an equation of state is not permitted for model {model}", line)
        elif model in (9, 10):
            if eos == 0:
                raise DeckError(f"material {n}: model {model} requires an equation of state", line)
            if eos not in _EOS_CARDS:
                raise DeckError("error in input - eos type not implemented", line)
        else:
            raise DeckError("error in input - material type not implemented", line)
        m = MaterialCard(model=model, eos=eos, rho=rho, visc_type=vt, av_l=avl, av_q=avq, mass=mass, h=h,
                         rho_min=rmin, rho_max=rmax, ihq=ihq, qh=qh)
        m.head = cards.next(" error reading material heading card")[:72].rstrip()
        ncard, per = _PROP_CARDS[model]
        for j in range(ncard):
            vals = cards.read(" error reading material property cards", "(8e10.0)", per)
            m.strinput[j * per:(j + 1) * per] = vals
        if eos != 0:
            m.eos_head = cards.next(" error reading eos property cards")[:72].rstrip()
            k = 0
            for cnt, fmt in _EOS_CARDS[eos]:
                vals = cards.read(" error reading eos property cards", fmt, cnt)
                m.eosinput[k:k + cnt] = vals
                k += cnt
        mats[n - 1] = m
    missing = [k + 1 for k, m in enumerate(mats) if m is None]
    if missing:
        raise DeckError(f"material cards define no material {missing[0]}", cards.line)
    return mats


def _nodes(cards: _Cards, d: dict) -> None:
    """MCM/mcm_nodein.f90:33-115."""
    ndim, n = d["ndim"], d["np"]
    x = np.zeros((n, 3))
    mat = np.zeros(n, dtype=np.int32)
    disp = np.zeros(n, dtype=np.int32)
    fmt = f"(i8,i5,{ndim}e20.0,i7)"
    # all cards at once when every field is a plain number and the cards are in
    # order; otherwise card by card, which applies the full rules and reports
    # the first bad card
    start = cards.pos
    texts, _ = cards.block(n)
    cols = _bulk_columns(texts, fmt) if len(texts) == n else None
    ok = (cols is not None and np.array_equal(cols[0], np.arange(1, n + 1))
          and bool(((cols[2 + ndim] > 0) & (cols[2 + ndim] <= d["nummat"])).all()))
    if ok:
        x[:, :ndim] = np.stack(cols[2:2 + ndim], axis=1)
        mat[:] = cols[2 + ndim]
        disp[:] = cols[1]
    else:
        cards.pos = start
        for j in range(1, n + 1):
            v = cards.read("Error in nodal poistion cards", fmt)
            if v[0] != j:
                cards.fail(f"Card for node {v[0]} is out of order. Should be {j}")
            disp[j - 1] = v[1]
            x[j - 1, :ndim] = v[2:2 + ndim]
            mat[j - 1] = v[2 + ndim]
            if mat[j - 1] == 0:
                cards.fail(f"Node {j} has zero material type")
            if not 0 < mat[j - 1] <= d["nummat"]:
                cards.fail(f"Node {j} has material {mat[j - 1]}, beyond the {d['nummat']} materials")
    d["x"], d["mat"], d["dispbc"] = x, mat, disp
    if d["massopt"] == 1 or d["init_h_opt"] == 1 or d["init_rhoe"] == 1:
        pd = np.zeros((n, 4))
        start = cards.pos
        texts, _ = cards.block(n)
        cols = _bulk_columns(texts, "(i8,4e20.0)") if len(texts) == n else None
        if cols is not None and np.array_equal(cols[0], np.arange(1, n + 1)):
            pd[:] = np.stack(cols[1:], axis=1)
            d["pardata"] = pd
            return
        cards.pos = start
        for j in range(1, n + 1):
            v = cards.read("Error in additional particle information cards", "(i8,4e20.0)")
            if v[0] != j:
                cards.fail(f"Additional information card for node {v[0]} is out of order. Should be {j}")
            pd[j - 1] = v[1:]
        d["pardata"] = pd


def read_thnodes(cards: _Cards, thnode: int, np_: int) -> tuple:
    """MCM/mcm_nodehist.f90:29-62.  Cards of 10i8; the reference stores item
    l of card i (i counted from 0) at position i + l (:43, :55), not 10 i + l,
    so with more than 10 particles the cards overlap and the last positions
    stay unset.  Up to 10 particles (one card) are read as the reference reads
    them; more raise DeckError."""
    if thnode <= 10:
        last, last1 = 0, thnode
    else:
        last, last1 = thnode // 10, thnode % 10
    ids = [0] * thnode
    written = [False] * thnode
    for i in range(last + 1):
        cnt = 10 if i < last else last1
        vals = cards.read(" error reading nodes for time histry", "(10i8)", cnt)
        for l, v in enumerate(vals, start=1):
            ids[i + l - 1] = v
            written[i + l - 1] = True
    if not all(written):
        raise DeckError(f"{thnode} time-history particles: the reference reads at most 10 "
                        "(MCM/mcm_nodehist.f90:43 stores card i item l at i+l)", cards.line)
    return tuple(ids)


def _velocities(cards: _Cards, d: dict) -> np.ndarray:
    """MCM/mcm_Inputvel.f90:32-108: a card (nid, v) with nid > i fills
    particles i..nid with v, which must equal the previous card's velocity."""
    ndim, n = d["ndim"], d["np"]
    v = np.zeros((n, 3))
    if d["init_v_opt"] != 1:
        return v
    fmt = f"(i8,{ndim}e10.0)"
    msg = "Error reading initial velocity cards"
    vals = cards.read(msg, fmt)
    if vals[0] != 1:
        cards.fail("Error, first nodal velocity card is not for node 1")
    v[0, :ndim] = vals[1:]
    gen, nid = False, 1
    for i in range(2, n + 1):
        if not gen:
            vals = cards.read(msg, fmt)
            nid = vals[0]
            v[i - 1, :ndim] = vals[1:]
            if nid > i:
                if nid > n:
                    cards.fail("Nodal id exceeds number of particles")
                for k, ax in enumerate("xyz"):
                    if v[i - 1, k] != v[i - 2, k]:
                        cards.fail(f"{ax} velocity for auto generation is not constant")
                gen = True
            elif nid < i:
                cards.fail("Nodal id is less than previous card")
        else:
            v[i - 1] = v[i - 2]
            if i == nid:
                gen = False
    return v


def _symmetry_v2(cards: _Cards, d: dict) -> None:
    """MCM/mcm_inp_symmetry_v2.f90:29-137 (flags 1 = symmetry, 2 = periodic)."""
    nd = 2 * d["ndim"]
    flags = cards.read("Error reading boundary plane flag card", "(6i10)", nd) + [0] * (6 - nd)
    xs = cards.read("Error reading boundary plane coordinate card", "(6e10.0)", nd) + [0.0] * (6 - nd)
    for i in range(0, 6, 2):
        if flags[i] == 2 and flags[i + 1] != 2:
            cards.fail(f"periodic plane {i + 1}: the corresponding maximum plane is not periodic")
        if flags[i + 1] == 2 and flags[i] != 2:
            cards.fail(f"periodic plane {i + 2}: the corresponding minimum plane is not periodic")
    d["sym_flag"], d["sym_x"] = tuple(flags), tuple(xs)


def _symmetry_v1(cards: _Cards, d: dict) -> None:
    """MCM/mcm_inp_symmetry_v1.f90:29-80: coordinates first, then one flag per
    plane where 0 (not 1) makes the plane a symmetry plane."""
    nd = 2 * d["ndim"]
    xs = cards.read("Error reading Symetry plans cards", "(6e10.0)", nd) + [0.0] * (6 - nd)
    fl = cards.read("Error reading Reflection plans cards", "(6i5)", nd)
    d["sym_flag"] = tuple(1 if (k < nd and fl[k] == 0) else 0 for k in range(6))
    d["sym_x"] = tuple(xs)


# ------------------------------------------------------------------ writing
def _r(x, w):
    return real_field(x, w)


def _i(n, w):
    return int_field(n, w)


def deck_text(deck: Deck, comments: bool = True) -> str:
    """Version-2 deck text of `deck` (the inverse of read_deck)."""
    out = io.StringIO()
    w = out.write
    ndim, n = deck.ndim, deck.np
    nummat = len(deck.materials)

    def note(s):
        if comments:
            w(f"$ {s}\n")

    title = (deck.title or deck.name)[:78]
    if title[:1] in ("*", "$"):
        title = " " + title[:77]
    w(f"{title:<78}{_i(2, 2)}\n")
    note("control cards (MCM/mcm_control_v2.f90)")
    w(_i(ndim, 5) + _i(deck.disctype, 5) + _i(nummat, 10) + _i(n, 10) + _i(deck.max_np, 10)
      + _i(deck.nstressp, 10) + _i(deck.nvelocp, 10) + "\n")
    w(_r(deck.endtime, 10) + _r(deck.tssf, 10) + _r(deck.itss, 10) + _r(deck.drelax_scale, 10) + "\n")
    w(_r(deck.stpltime, 10) + _i(deck.state_opt, 5) + _r(deck.thpltime, 10) + _i(len(deck.thnodes), 10)
      + _i(len(deck.transducers), 5) + _i(deck.status_interval, 10) + _i(deck.restart_interval, 5)
      + _i(deck.run_restart, 5) + "\n")
    w("".join(_i(k, 5) for k in (deck.keep_files, deck.init_v_opt, deck.massopt, deck.init_h_opt,
                                 deck.init_rhoe)) + "\n")
    w("".join(_i(k, 5) for k in (deck.contacttype, deck.tcrit_opt, deck.veloc_opt, deck.mirr_opt, deck.nlcur,
                                 *deck.nthp)) + "\n")
    w(_i(deck.h_opt, 5) + _i(deck.krtype, 5) + _i(deck.maxnbr, 5) + "\n")
    w(_i(0, 5) + "\n")
    for k, m in enumerate(deck.materials, start=1):
        note(f"material {k} (MCM/mcm_matin.f90)")
        w(_i(k, 5) + _i(m.model, 5) + _r(m.rho, 10) + _i(m.eos, 5) + _i(m.ihq, 5) + _r(m.qh, 10)
          + _i(m.visc_type, 5) + _r(m.av_q, 10) + _r(m.av_l, 10) + "\n")
        w(_r(m.mass, 10) + _r(m.h, 10) + _r(m.rho_min, 10) + _r(m.rho_max, 10) + "\n")
        w(_heading(m.head, f"material {k} model {m.model}"))
        if m.model not in _PROP_CARDS:
            raise ValueError(f"material model {m.model} has no property-card layout")
        ncard, per = _PROP_CARDS[m.model]
        for j in range(ncard):
            w("".join(_r(x, 10) for x in m.strinput[j * per:(j + 1) * per]) + "\n")
        if m.eos != 0:
            w(_heading(m.eos_head, f"eos {m.eos}"))
            kk = 0
            for cnt, _ in _EOS_CARDS[m.eos]:
                w("".join(_r(x, 10) for x in m.eosinput[kk:kk + cnt]) + "\n")
                kk += cnt
    note("nodes (MCM/mcm_nodein.f90: i8, i5, 3e20.0, i7)")
    x = np.asarray(deck.x, dtype=np.float64)
    disp = np.zeros(n, dtype=np.int64) if deck.dispbc is None else np.asarray(deck.dispbc)
    mat = np.asarray(deck.mat)
    lines = []
    for j in range(n):
        lines.append(_i(j + 1, 8) + _i(disp[j], 5) + "".join(_r(x[j, k], 20) for k in range(ndim))
                     + _i(mat[j], 7) + "\n")
    w("".join(lines))
    if deck.massopt == 1 or deck.init_h_opt == 1 or deck.init_rhoe == 1:
        if deck.pardata is None:
            raise ValueError("massopt/init_h_opt/init_rhoe = 1 needs deck.pardata (mass, h, rho, e)")
        pd = np.asarray(deck.pardata, dtype=np.float64)
        note("additional particle data: mass, h, rho, e")
        # (i8,4e20.0) spans 88 columns of an 80-column record (MCM/mcm_gttxsg.f90:33
        # reads a80): the energy must sit in the first 12 columns of its field
        w("".join(_i(j + 1, 8) + "".join(_r(pd[j, k], 20) for k in range(3)) + _r(pd[j, 3], 12) + "\n"
                  for j in range(n)))
    if deck.thnodes:
        if len(deck.thnodes) > 10:
            raise ValueError("the reference reads at most 10 time-history particles (MCM/mcm_nodehist.f90:43)")
        note("time-history particles")
        w("".join(_i(t, 8) for t in deck.thnodes) + "\n")
    for pos, m in deck.transducers:
        w("".join(_r(pos[k], 10) for k in range(ndim)) + _i(m, 5) + "\n")
    if deck.init_v_opt == 1:
        note("initial velocities (MCM/mcm_Inputvel.f90: a card nid > i fills i..nid)")
        w("".join(_velocity_cards(np.asarray(deck.v, dtype=np.float64), ndim)))
    if deck.mirr_opt == 1:
        note("boundary planes: xmin xmax ymin ymax zmin zmax (1 symmetry, 2 periodic)")
        w("".join(_i(f, 10) for f in deck.sym_flag[:2 * ndim]) + "\n")
        w("".join(_r(s, 10) for s in deck.sym_x[:2 * ndim]) + "\n")
    if deck.contacttype > 0:
        w(_i(deck.ncontmats, 5) + _i(deck.cont_opt, 5) + "\n")
        if deck.ncontmats == -1:
            for k in range(nummat):
                w(_r(deck.k_cont[k], 10) + _r(deck.n_cont[k], 10) + "\n")
    if any(t == 1 for t in deck.nthp):
        note("base accelerations")
        w("".join(_r(a, 20) for a in deck.base_a) + "\n")
    text = out.getvalue()
    long = [k for k, ln in enumerate(text.splitlines(), 1) if len(ln) > 80]
    if long:
        raise AssertionError(f"deck lines {long[:3]} exceed 80 columns")
    return text


def _heading(text: str, default: str) -> str:
    t = (text or default)[:72]
    if t[:1] in ("*", "$"):
        t = " " + t[:71]
    return t + "\n"


def _velocity_cards(v: np.ndarray, ndim: int) -> list:
    """Runs of equal velocities become a first card and a generation card.
    What is equal is the text a velocity has in the deck: runs of equal
    doubles are found first, then neighbouring runs whose text is the same
    are joined."""
    n = v.shape[0]
    if n == 0:
        return []
    vv = v[:, :ndim]
    starts = np.flatnonzero(np.concatenate([[True], np.any(vv[1:] != vv[:-1], axis=1)]))
    ends = np.concatenate([starts[1:], [n]]) - 1
    runs = []                      # (first, last, text)
    for a, b in zip(starts.tolist(), ends.tolist()):
        txt = "".join(_r(vv[a, k], 10) for k in range(ndim))
        if runs and runs[-1][2] == txt:
            runs[-1] = (runs[-1][0], b, txt)
        else:
            runs.append((a, b, txt))
    cards = []
    for a, b, txt in runs:
        cards.append(_i(a + 1, 8) + txt + "\n")
        if b > a:
            cards.append(_i(b + 1, 8) + txt + "\n")
    return cards


def write_deck(deck: Deck, path, comments: bool = True) -> None:
    with open(path, "w") as f:
        f.write(deck_text(deck, comments))
