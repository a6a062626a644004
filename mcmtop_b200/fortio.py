"""Fortran formatted-record reading and writing, as MCM's deck reader and
output writers use it.

MCM reads every input card into an 80-character string (``read(fmt='(a80)')``
in MCM/mcm_gttxsg.f90:33, format 20) and then decodes fixed-width fields from
it with internal READs such as ``(2i5,5i10)`` (MCM/mcm_control_v2.f90:274) or
``(i8,i5,3e20.0,i7)`` (MCM/mcm_nodein.f90:155).  Its writers produce fixed-
width records (``F15.8``, ``E24.5``, ``e14.6``, ``I5``).  This module restates
the edit-descriptor rules of the Fortran standard for those cases:

* input Iw: blanks are ignored (BLANK='NULL', the default of an internal
  file), an all-blank field is zero;
* input Fw.d / Ew.d / Dw.d: optional sign, digits with an optional decimal
  point, optional exponent written as E/D/Q followed by a signed integer or as
  a bare signed integer; without a decimal point the last d digits are the
  fraction; blanks are ignored; the decimal value is rounded to the nearest
  double;
* output Iw, Fw.d, Ew.d: right-justified, ``*`` characters filling the field
  when the value does not fit, E editing as ``0.ddddE+xx`` (a three-digit
  exponent drops the letter), the optional leading zero written when there is
  room.  Decimal digits are the correctly rounded digits of the binary value
  (ties to even).
"""
from __future__ import annotations

import re
from decimal import Decimal

RECORD = 80   # MCM/mcm_gttxsg.f90:33 reads records as a80

_REAL = re.compile(r"^([+-]?)(\d*)(\.?)(\d*)(?:[EeDdQq]([+-]?\d+)|([+-]\d+))?$")
_INT = re.compile(r"^[+-]?\d+$")


class FieldError(ValueError):
    """A field that an internal Fortran READ would reject (err= branch)."""


def parse_format(fmt: str) -> list:
    """'(2i5,e10.0,3e20.0)' -> [('i', 5, 0), ('i', 5, 0), ('e', 10, 0), ...].

    Only repeat counts and the I, E, F, D and A descriptors occur in MCM's
    card formats; parentheses groups are not needed."""
    out = []
    body = fmt.strip()
    if body.startswith("(") and body.endswith(")"):
        body = body[1:-1]
    for item in body.split(","):
        m = re.fullmatch(r"\s*(\d*)([iefdaIEFDA])(\d+)(?:\.(\d+))?\s*", item)
        if not m:
            raise ValueError(f"unsupported edit descriptor {item!r}")
        rep = int(m.group(1) or 1)
        kind = m.group(2).lower()
        if kind == "d":
            kind = "e"
        if kind == "f":
            kind = "e"
        out.extend([(kind, int(m.group(3)), int(m.group(4) or 0))] * rep)
    return out


def read_int(field: str) -> int:
    s = field.replace(" ", "")
    if not s:
        return 0
    if not _INT.match(s):
        raise FieldError(f"bad integer field {field!r}")
    return int(s)


def read_real(field: str, d: int = 0) -> float:
    s = field.replace(" ", "")
    if not s:
        return 0.0
    m = _REAL.match(s)
    if not m or (m.group(2) == "" and m.group(4) == ""):
        raise FieldError(f"bad real field {field!r}")
    sign, ip, dot, fp, e1, e2 = m.groups()
    exp = int(e1 or e2 or 0)
    if dot:
        digits, scale = ip + fp, -len(fp)
    else:
        digits, scale = ip, -d
    return float(f"{sign}{digits or '0'}e{exp + scale}")


def read_record(record: str, fmt, count: int | None = None) -> list:
    """Decodes the first `count` items (all by default) of an 80-column record
    with the given format, as ``read(unit=record, fmt=fmt) items`` does.  The
    record is cut at 80 columns and padded with blanks; items beyond the end
    of the format's list are not read."""
    spec = parse_format(fmt) if isinstance(fmt, str) else fmt
    if count is not None:
        spec = spec[:count]
    rec = record.rstrip("\r\n")[:RECORD].ljust(RECORD)
    out, pos = [], 0
    for kind, w, d in spec:
        field = rec[pos:pos + w] if pos < len(rec) else ""
        pos += w
        if kind == "i":
            out.append(read_int(field))
        elif kind == "e":
            out.append(read_real(field, d))
        else:
            out.append(field)
    return out


# ---------------------------------------------------------------- output
def fmt_i(n: int, w: int) -> str:
    s = str(int(n))
    return s.rjust(w) if len(s) <= w else "*" * w


def fmt_f(x: float, w: int, d: int) -> str:
    x = float(x)
    if x != x or x in (float("inf"), float("-inf")):
        s = "NaN" if x != x else ("Infinity" if x > 0 else "-Infinity")
        return s.rjust(w) if len(s) <= w else "*" * w
    s = f"{x:.{d}f}"
    if len(s) > w:
        # the leading zero of |x| < 1 is optional
        if s.startswith("0."):
            s = s[1:]
        elif s.startswith("-0."):
            s = "-" + s[2:]
    return s.rjust(w) if len(s) <= w else "*" * w


def fmt_e(x: float, w: int, d: int) -> str:
    x = float(x)
    if x != x or x in (float("inf"), float("-inf")):
        s = "NaN" if x != x else ("Infinity" if x > 0 else "-Infinity")
        return s.rjust(w) if len(s) <= w else "*" * w
    neg = x < 0 or (x == 0.0 and str(x).startswith("-"))
    if x == 0.0:
        digits, exp = "0" * d, 0
    else:
        # d significant digits: 0.d1d2...dd x 10^exp
        m = f"{abs(x):.{d - 1}e}" if d > 0 else f"{abs(x):.0e}"
        mant, e = m.split("e")
        digits = mant.replace(".", "")[:d] if d > 0 else ""
        exp = int(e) + 1
    if abs(exp) <= 99:
        es = f"E{'-' if exp < 0 else '+'}{abs(exp):02d}"
    elif abs(exp) <= 999:
        es = f"{'-' if exp < 0 else '+'}{abs(exp):03d}"
    else:
        return "*" * w
    body = f".{digits}{es}"
    s = ("-" if neg else "") + "0" + body
    if len(s) > w:
        s = ("-" if neg else "") + body
    return s.rjust(w) if len(s) <= w else "*" * w


# ------------------------------------------------------- deck-field writing
def _compact(s: str) -> str:
    """'1.5e-05' -> '1.5e-5'; '2e+03' -> '2.e3' (a decimal point always present)."""
    if "e" in s:
        mant, e = s.split("e")
        if "." not in mant:
            mant += "."
        return f"{mant}e{int(e)}"
    return s if "." in s else s + "."


def _renderings(x: float):
    """Exact texts of x built from its shortest round-trip digits: fixed,
    fixed without the leading zero, scientific."""
    d = Decimal(repr(x))
    f = format(d, "f")
    f = f.rstrip("0") if "." in f else f + "."
    yield f
    if f.startswith("0.") or f.startswith("-0."):
        yield f.replace("0.", ".", 1)
    sign, digits, exp = d.as_tuple()
    ds = "".join(map(str, digits)).rstrip("0") or "0"
    e = exp + len(digits) - 1
    yield ("-" if sign else "") + ds[0] + "." + ds[1:] + f"e{e}"


def real_field(x: float, w: int) -> str:
    """Text for x in a w-column real input field, read back with any Ew.d or
    Fw.d because it always holds a decimal point, and leaving the first
    column blank so that adjacent fields stay apart.  The value written is
    the one nearest to x among the fixed and scientific forms that fit; its
    text is then the first of its exact renderings that fits, so writing the
    value read back gives the same text."""
    x = float(x)
    room = w - 1
    if x == 0.0:
        return "0.0".rjust(w)
    if x != x or x in (float("inf"), float("-inf")):
        raise ValueError(f"{x!r} has no deck representation")
    r = repr(x)
    if "e" not in r:
        # the first rendering without building a Decimal: repr's positional digits
        f = r.rstrip("0") if "." in r else r + "."
        if len(f) <= room:
            return f.rjust(w)
    for t in _renderings(x):
        if len(t) <= room:
            return t.rjust(w)
    cands = []
    for p in range(min(17, room), -1, -1):
        c = _compact(f"{x:.{p}e}")
        if len(c) <= room:
            cands.append(c)
            break
    if abs(x) < 10.0 ** room:
        for p in range(min(24, room), -1, -1):
            c = f"{x:.{p}f}" + ("." if p == 0 else "")
            if c.startswith("0.") or c.startswith("-0."):
                c = c.replace("0.", ".", 1)
            if len(c) <= room and c not in (".", "-.") and float(c) != 0.0:
                cands.append(c)
                break
    if not cands:
        raise ValueError(f"{x!r} does not fit a {w}-column real field")
    xv = float(min(cands, key=lambda c: abs(float(c) - x)))
    for t in _renderings(xv):
        if len(t) <= room:
            return t.rjust(w)
    raise AssertionError(f"no rendering of {xv!r} fits {room} columns")


def int_field(n: int, w: int) -> str:
    s = str(int(n))
    if len(s) > w:
        raise ValueError(f"{n} does not fit a {w}-column integer field")
    return s.rjust(w)
