"""MCM's output files, written from the state downloaded at output times.

The GPU step leaves the Fortran-side writers unchanged; this module is the
same set of writers for a host program driving the step from Python:

* state files of output option 4 (legacy VTK): MCM/mcm_VTK.f90 ``WriteVTK``
  (all particles, ``<out><n>.vtk``) and ``WriteVTKmat`` (materials 1 and 2,
  ``<m><out><n>.vtk``, with the cap-model point type), called by
  MCM/mcm_init_state_output.f90:61-66 and MCM/mcm_state_output.f90:89-93;
* time histories: MCM/mcm_inittimehist.f90 (file headers) and
  MCM/mcm_timehist.f90 (``<out>_thist.csv``: per-material energies and
  contact forces; ``<out>_th<id>.csv``: one particle's state);
* pressure transducers: MCM/mcm_transducer_nbr.f90 (particles of the
  transducer's material within 2h) and MCM/mcm_pressure_transducer.f90
  (SPH interpolation of pressure and velocity, ``<out>_ptrn.csv``,
  ``<out>_vtrn.csv``);
* the relaxed state after a dynamic-relaxation run: MCM/mcm_write_drelax.f90
  (``<out>.drlx``).

Record layouts, number formats (fortio.fmt_e / fmt_f / fmt_i) and the
values zeroed below 1e-50 (1e-40 for transducers) follow those routines.
Deliberate differences: where the reference's integer fields overflow
(``I5`` point counts from 100 000 particles, ``I6`` cell ids from 1 000 000,
``I3`` state numbers from 1 000) it writes asterisks that no reader accepts;
these writers widen the field instead.  The state writers of options 2-3
(EnSight case, LS-DYNA d3plot) and the 1D/2D ASCII state plots of option 0 are
not provided: option 0 has no writer for 3D problems in the reference
either (MCM/mcm_Stateplot.f90:40-47).  Option 1 (EnSight: geometry at the
start, 21 variable files per state, results file, time file) follows
MCM/mcm_geometry.f90, MCM/mcm_write_ensight_3d.f90 with
MCM/mcm_write_scalar.f90 / mcm_write_vector.f90 / mcm_write_tensor.f90, and
MCM/mcm_write_res.f90.
"""
from __future__ import annotations

import math
import os

import numpy as np

from .fortio import fmt_e, fmt_f, fmt_i, read_real

# fields a state or time-history record reads
VTK_FIELDS = ("x", "v", "p", "sigma", "mat", "ptype")
TH_FIELDS = ("x", "v", "rho", "p", "sigma", "efps", "e", "mass", "c", "critts")
TR_FIELDS = ("x", "v", "mass", "rho", "p", "h", "mat")

_TH_HEAD_3D = (",Time,x coordinate,y coordinate,z coordinate,x velocity,y velocity,z velocity,"
               "Density,Pressure,11 Stress,22 Stress,33 Stress,12 Stress,13 Stress,23 Stress,"
               " Eff. Plastic Strain,Total Internal Energy,Speed of Sound,Critical timestep,Temperature")


def _count(n: int) -> str:
    """charParNumb of MCM/mcm_VTK.f90:45-56: the count left-aligned in 25
    characters (I1..I5 by magnitude), widened past 99 999."""
    return f"{n:<25d}"


def _vm_stress(sig: np.ndarray) -> np.ndarray:
    """VMStress of MCM/mcm_VTK.f90:153-158: the FP64 expression in the
    reference's order, stored in a default REAL (FP32) variable."""
    s11, s22, s33 = sig[:, 0, 0], sig[:, 1, 1], sig[:, 2, 2]
    s12, s23, s13 = sig[:, 0, 1], sig[:, 1, 2], sig[:, 0, 2]
    a = (s11 - s22) * (s11 - s22) + (s22 - s33) * (s22 - s33)
    a = a + (s33 - s11) * (s33 - s11)
    b = s12 * s12 + s23 * s23
    b = b + s13 * s13
    return np.sqrt(0.5 * (a + 6.0 * b)).astype(np.float32)


def vtk_text(state: dict, sel: np.ndarray | None = None, with_ptype: bool = False) -> str:
    """One legacy-VTK state file: WriteVTK (sel None, all particles) or
    WriteVTKmat (sel = the particles of one material, with_ptype True)."""
    x, v, p, sig = state["x"], state["v"], state["p"], state["sigma"]
    if sel is not None:
        x, v, p, sig = x[sel], v[sel], p[sel], sig[sel]
    n = x.shape[0]
    out = ["# vtk DataFile Version 3.0\n", "TEST\n", "ASCII\n", "DATASET UNSTRUCTURED_GRID\n",
           f" POINTS {_count(n)} double\n"]
    out.extend(fmt_f(a, 15, 8) + fmt_f(b, 15, 8) + fmt_f(c, 15, 8) + "\n" for a, b, c in x.tolist())
    out.append(f" CELLS {_count(n)} {_count(2 * n)}\n")
    out.extend(f"1 {k:6d}\n" for k in range(n))
    out.append(f"CELL_TYPES {n:5d}\n")
    out.append("1\n" * n)
    out.append(f"POINT_DATA {n:5d}\n")
    out.append(" VECTORS Velocities double\n")
    out.extend(fmt_f(a, 15, 8) + fmt_f(b, 15, 8) + fmt_f(c, 15, 8) + "\n" for a, b, c in v.tolist())

    def scalars(name, vals):
        out.append(f"SCALARS {name} double 1\n")
        out.append("LOOKUP_TABLE default\n")
        out.extend(fmt_e(a, 24, 5) + "\n" for a in vals.tolist())

    scalars("Pressure", p)
    scalars("Stress_X", sig[:, 0, 0])
    scalars("Stress_Y", sig[:, 1, 1])
    scalars("Stress_Z", sig[:, 2, 2])
    scalars("Shear_Stress_XY", sig[:, 0, 1])
    scalars("Shear_Stress_XZ", sig[:, 0, 2])
    scalars("Shear_Stress_YZ", sig[:, 1, 2])
    scalars("VM_Stress", _vm_stress(sig).astype(np.float64))
    if with_ptype:
        pt = state["ptype"] if sel is None else state["ptype"][sel]
        out.append("SCALARS PTYPE double 1\n")
        out.append("LOOKUP_TABLE default\n")
        out.extend(f"{int(a):5d}\n" for a in pt.tolist())
    return "".join(out)


def read_vtk(path: str) -> dict:
    """Parses a file written by vtk_text back into arrays (for checks)."""
    with open(path) as f:
        lines = f.read().split("\n")
    out, i = {}, 0
    while i < len(lines):
        t = lines[i].split()
        if not t:
            i += 1
            continue
        if t[0] == "POINTS":
            n = int(t[1])
            out["x"] = np.array([[float(s) for s in lines[i + 1 + k].split()] for k in range(n)]).reshape(n, 3)
            i += n + 1
        elif t[0] == "VECTORS":
            n = out["x"].shape[0]
            out["v"] = np.array([[float(s) for s in lines[i + 1 + k].split()] for k in range(n)]).reshape(n, 3)
            i += n + 1
        elif t[0] == "SCALARS":
            n = out["x"].shape[0]
            out[t[1]] = np.array([float(lines[i + 2 + k]) for k in range(n)])
            i += n + 2
        else:
            i += 1
    return out


class Outputs:
    """Output cadence and files of MCM/mcm_initial.f90:109-115 and
    MCM/mcm_solution.f90:81-92 for one problem.

    ``fileout`` is the output base name (MCM's ``o=`` argument), ``directory``
    where the files go."""

    def __init__(self, deck, fileout: str, directory: str = "."):
        self.deck = deck
        self.base = os.path.join(directory, fileout)
        self.title = (deck.title or deck.name)[:78]
        self.nummat = len(deck.materials)
        self.istate = 0
        self.nextsttime = 0.0
        self.nextthtime = 0.0
        self.files = []

    # --------------------------------------------------------- cadence
    def fields(self, state_due: bool, th_due: bool) -> tuple:
        need = set()
        if state_due and self.deck.state_opt == 4:
            need.update(VTK_FIELDS)
        if state_due and self.deck.state_opt == 1:
            need.update(ENSIGHT_FIELDS)
        if th_due:
            if self.deck.thnodes:
                need.update(TH_FIELDS)
            if self.deck.transducers:
                need.update(TR_FIELDS)
        return tuple(sorted(need))

    def due(self, ptime: float) -> tuple:
        end = self.deck.endtime
        return ptime >= self.nextsttime or ptime >= end, ptime >= self.nextthtime or ptime >= end

    def next_time(self) -> float:
        return min(self.nextsttime, self.nextthtime, self.deck.endtime)

    def initial(self, ptime: float, state: dict, energies: np.ndarray) -> None:
        """mcm_init_state_output + mcm_state_output, mcm_inittimehist + mcm_timehist."""
        self.nextsttime = ptime + self.deck.stpltime
        self.ptime = ptime
        if self.deck.state_opt == 4:
            self._write_vtk(state)          # MCM/mcm_init_state_output.f90:61-64 (no increment)
        if self.deck.state_opt == 1:
            # MCM/mcm_init_state_output.f90:28-32: the counter starts at 1, mcm_geometry
            # writes the initial coordinates and clears the time file
            self.istate = 1
            self.times = []
            self._put(self.base + ".geo", ensight_geometry_text(state["x"], state["mat"], self.nummat))
            self._put(self.base + "_time.txt", "")
        self.state_output(state)
        self.nextthtime = ptime + self.deck.thpltime
        self._init_timehist()
        self.timehist(ptime, state, energies)

    def after_energies(self, ptime: float, state: dict, energies: np.ndarray, contact_forces=None) -> None:
        """MCM/mcm_solution.f90:81-92, called after mcm_calctotale; contact_forces
        (nmat, 3) are the step's mcm_mat%xcf, %ycf, %zcf (zero when omitted)."""
        st, th = self.due(ptime)
        self.ptime = ptime
        if st:
            self.state_output(state)
            self.nextsttime += self.deck.stpltime
        if th:
            self.timehist(ptime, state, energies, contact_forces)
            self.nextthtime += self.deck.thpltime

    # ---------------------------------------------------------- states
    def state_output(self, state: dict) -> None:
        """MCM/mcm_state_output.f90: option 4 writes the VTK files, option 1
        the EnSight variable files and the results file; both count."""
        if self.deck.state_opt == 4:
            self._write_vtk(state)
            self.istate += 1
        elif self.deck.state_opt == 1:
            self._write_ensight(state)
            self.istate += 1

    def _write_ensight(self, state: dict) -> None:
        """MCM/mcm_write_ensight_3d.f90 then MCM/mcm_write_res.f90."""
        t = fmt_e(self.ptime, 13, 6)
        self.times.append(t)
        self._put(self.base + "_time.txt", t + "\n", "a")
        ext = f"{self.istate:03d}" if self.istate < 1000 else str(self.istate)
        x0 = np.asarray(self.deck.x, dtype=np.float64)   # xzero: the deck's coordinates (MCM/mcm_initvbls.f90:32)
        for suf, head, kind, vals in _ensight_variables(state, x0):
            body = _ens_vector(vals) if kind == "v" else _ens_scalar(vals)
            self._put(self.base + suf + ext, " " + head + "\n" + "".join(body))
        name = os.path.basename(self.base)
        self._put(self.base + ".res", ensight_res_text(name, self.istate, self.times))

    def _write_vtk(self, state: dict) -> None:
        d, name = os.path.split(self.base)
        tag = f"{self.istate:d}.vtk"
        path = os.path.join(d, name + tag)
        self._put(path, vtk_text(state))
        for m in (1, 2):                     # MCM/mcm_state_output.f90:91-92
            sel = np.flatnonzero(state["mat"] == m)
            self._put(os.path.join(d, f"{m:d}{name}{tag}"), vtk_text(state, sel, with_ptype=True))

    def drelax(self, state: dict) -> None:
        """MCM/mcm_write_drelax.f90: written once, after the loop, when
        dynamic relaxation is active (0.1 < drelax_scale < 1)."""
        if 0.1 < self.deck.drelax_scale < 1.0:
            self._put(self.base + ".drlx", drelax_text(state))

    def _put(self, path: str, text: str, mode: str = "w") -> None:
        with open(path, mode) as f:
            f.write(text)
        if path not in self.files:
            self.files.append(path)

    # ---------------------------------------------------- time history
    def _th_path(self, pid: int) -> str:
        # MCM/mcm_inittimehist.f90:62-65: '_th' // I<digits> // '.csv'
        return f"{self.base}_th{pid:d}.csv"

    def _init_timehist(self) -> None:
        title = f"{self.title:<78}\n"
        self._put(self.base + "_thist.csv", title + "Global time history data\n")
        for pid in self.deck.thnodes:
            if pid <= 0:
                raise ValueError(f"time-history particle id {pid} is not positive")
            self._put(self._th_path(pid), title + f"Time history data for particle {pid:6d}\n"
                      + _TH_HEAD_3D + "\n")
        if self.deck.transducers:
            self._put(self.base + "_ptrn.csv", title + "Time,Pressure transducer time histories\n")
            self._put(self.base + "_vtrn.csv", title + "Time,Velocity transducer time histories\n")

    def timehist(self, ptime: float, state: dict, energies: np.ndarray, contact_forces=None) -> None:
        """MCM/mcm_timehist.f90:41-64 and the 3D rows of :112-140.  The contact
        forces of each material (xcf, ycf, zcf) are zero before the first
        momentum sum and without repulsive contact."""
        row = [ptime]
        cf = np.zeros((self.nummat, 3)) if contact_forces is None else np.asarray(contact_forces)
        for m in range(self.nummat):
            ke, ie = energies[5 * m], energies[5 * m + 1]
            row += [ke, ie, float(cf[m, 0]), float(cf[m, 1]), float(cf[m, 2])]
        self._put(self.base + "_thist.csv", "".join("," + fmt_e(a, 14, 6) for a in row) + "\n", "a")
        if self.deck.transducers:
            self._transducers(ptime, state)
        for pid in self.deck.thnodes:
            i = pid - 1
            s = state["sigma"][i]
            cols = [*state["x"][i], *state["v"][i], state["rho"][i], state["p"][i], s[0, 0], s[1, 1], s[2, 2],
                    s[0, 1], s[0, 2], s[1, 2], state["efps"][i], state["e"][i] / state["mass"][i],
                    state["c"][i], state["critts"][i], 0.0]
            cols = [0.0 if abs(c) < 1.0e-50 else float(c) for c in cols]
            self._put(self._th_path(pid), "," + "".join(fmt_e(a, 14, 6) + "," for a in [ptime] + cols) + "\n",
                      "a")

    def _transducers(self, ptime: float, state: dict) -> None:
        """MCM/mcm_transducer_nbr.f90:46-86 and MCM/mcm_pressure_transducer.f90:28-80:
        particles of the transducer's material closer than 2h, summed only when
        more than one is found.  (The reference keeps at most maxnbr+10 of
        them and then reads past its list; all are summed here.)"""
        x, h = state["x"], state["h"]
        vol = state["mass"] / state["rho"]
        pres, vel = [], []
        for pos, mat in self.deck.transducers:
            r2 = ((x - np.asarray(pos)) ** 2).sum(axis=1)
            (idx,) = np.nonzero((r2 < (2.0 * h) ** 2) & (state["mat"] == mat))
            pi, vi = 0.0, np.zeros(3)
            if idx.size > 1:
                for j in idx:
                    w = _kernel_w(math.sqrt(r2[j]), h[j])
                    pi += vol[j] * state["p"][j] * w
                    vi += vol[j] * state["v"][j] * w
            pres.append(0.0 if abs(pi) < 1.0e-40 else pi)
            vel.extend(0.0 if abs(c) < 1.0e-40 else float(c) for c in vi)
        self._put(self.base + "_ptrn.csv", "".join(fmt_e(a, 14, 6) + "," for a in [ptime] + pres) + "\n", "a")
        self._put(self.base + "_vtrn.csv", "".join(fmt_e(a, 14, 6) + "," for a in [ptime] + vel) + "\n", "a")


def _kernel_w(r: float, h: float) -> float:
    """Cubic spline of MCM/mcm_kernel.f90:60-93 in 3D (c1 = 1/(pi h^3))."""
    c1 = 1.0 / (math.acos(-1.0) * h * h * h)
    z = r / h
    if z < 1.0:
        return c1 * ((0.75 * z - 1.5) * z * z + 1.0)
    if z < 2.0:
        return 0.25 * c1 * (2.0 - z) ** 3
    return 0.0


# ----------------------------------------------------- EnSight (option 1)
ENSIGHT_FIELDS = ("x", "v", "a", "p", "rho", "mass", "sigma", "efps", "e", "c", "critts", "h", "nnbr", "mat")


def _e12(vals) -> str:
    return "".join(fmt_e(v, 12, 5) for v in vals)


def _zeroed(a: np.ndarray) -> np.ndarray:
    return np.where(np.abs(a) < 1.0e-50, 0.0, a)


def _ens_scalar(values: np.ndarray) -> list:
    """MCM/mcm_write_scalar.f90: six values per record (6(e12.5)), the last
    record holding what is left."""
    v = _zeroed(np.asarray(values, dtype=np.float64)).tolist()
    return [_e12(v[k:k + 6]) + "\n" for k in range(0, len(v), 6)]


def _ens_vector(values: np.ndarray) -> list:
    """MCM/mcm_write_vector.f90: two particles (six values) per record; the
    particles go in groups of six, the last group holding what is left."""
    v = _zeroed(np.asarray(values, dtype=np.float64))
    out = []
    for g in range(0, v.shape[0], 6):
        blk = v[g:g + 6]
        for k in range(0, blk.shape[0], 2):
            out.append(_e12(blk[k:k + 2].ravel().tolist()) + "\n")
    return out


def ensight_geometry_text(x: np.ndarray, mat: np.ndarray, nummat: int) -> str:
    """MCM/mcm_geometry.f90 (3D): coordinates, then per material the point
    numbers ind .. ind + count - 1 (consecutive, as if the particles were
    ordered by material)."""
    out = [" frame geometry\n", " node id assign\n", " element id assign\n", " coordinates\n", f"{len(x):7d}\n"]
    out.extend(_e12(r) + "\n" for r in x.tolist())
    ind = 1
    for j in range(1, nummat + 1):
        cnt = int((mat == j).sum())
        out.append(f"part {fmt_i(j, 1)}\n")
        out.append(f"points list of part {fmt_i(j, 1)}\n")
        out.append(" point\n")
        out.append(f"{cnt:8d}\n")
        out.extend(f"{k:8d}\n" for k in range(ind, ind + cnt))
        ind += cnt
    return "".join(out)


# (file suffix, header, value) of MCM/mcm_write_ensight_3d.f90, in the order the files are written
def _ensight_variables(st: dict, x0: np.ndarray) -> list:
    sig = st["sigma"]
    z = np.zeros(len(st["x"]))
    return [
        ("_displace", "displacement", "v", st["x"] - x0),
        ("_pressure", "pressure", "s", st["p"]),
        ("_velocity", "velocity", "v", st["v"]),
        ("_accelera", "acceleration", "v", st["a"]),
        ("_density", "density", "s", st["rho"]),
        ("_mass", "mass", "s", st["mass"]),
        ("_sigma11", "sigma11", "s", sig[:, 0, 0]),
        ("_sigma22", "sigma22", "s", sig[:, 1, 1]),
        ("_sigma33", "sigma33", "s", sig[:, 2, 2]),
        ("_sigma12", "sigma12", "s", sig[:, 0, 1]),
        ("_sigma13", "sigma13", "s", sig[:, 0, 2]),
        ("_sigma23", "sigma23", "s", sig[:, 1, 2]),
        ("_strain", "Effective plastic strain", "s", st["efps"]),
        ("_energy", "energy", "s", st["e"] / st["mass"]),
        ("_C", "C", "s", st["c"]),
        ("_PCT", "Partical_Critical_Timestep", "s", st["critts"]),
        ("_Temp", "Temperature", "s", z),                      # temper: not computed
        ("_Bound", "Boundary_Particles", "s", z),               # mcm_id_boundary is never called
        ("_Smooth", "Smoothing_length", "s", st["h"]),
        ("_Neigh", "Number_of_Neighbours", "s", st["nnbr"].astype(np.float64)),
        ("_material", "Material", "s", st["mat"].astype(np.float64)),
    ]


_RES_NAMES = [("_density", " density"), ("_pressure", " pressure"), ("_material", " material"), ("_mass", " mass"),
              ("_sigma11", " sigma11"), ("_sigma22", " sigma22"), ("_sigma12", " sigma12"), ("_sigma33", " sigma33"),
              ("_sigma13", " sigma13"), ("_sigma23", " sigma23"), ("_energy", " Internal_Energy"),
              ("_strain", " Eff_Plastic_Strain"), ("_C", " Sound Speed"), ("_PCT", " Part_Crit_Timestep"),
              ("_Temp", " Temperature"), ("_Bound", " Boundary_Particles"), ("_Smooth", " Smoothing_length"),
              ("_Neigh", " Nber_of_Neigbours"), ("_displace", " displacement"), ("_velocity", " velocity"),
              ("_accelera", " acceleration")]


def ensight_res_text(name: str, istate: int, times: list) -> str:
    """MCM/mcm_write_res.f90 (3D) before the state counter moves on: it lists
    istate - 1 times (the ones before the state just written), read back from
    the time file (so rounded to its e13.6) and written six per record with
    e10.3."""
    out = [" 18 3 0\n", f"{fmt_i(istate - 1, 3)}\n"]
    vals = [read_real(t) for t in times[:max(istate - 1, 0)]]
    for k in range(0, len(vals), 6):
        out.append("".join(fmt_e(v, 10, 3) for v in vals[k:k + 6]) + "\n")
    out.append(" 1 1\n")
    out.extend(f" {name}{suf}***{label}\n" for suf, label in _RES_NAMES)
    return "".join(out)


DRELAX_FIELDS = ("x", "dispbc", "mat", "mass", "h", "rho", "e")


def drelax_text(state: dict) -> str:
    """The relaxed state file of MCM/mcm_write_drelax.f90:36-72 (3D): node
    cards (i8,i5,3e20.13,i7) and additional particle cards (i8,4e20.13), the
    layouts of MCM/mcm_nodein.f90 so that the lines can be pasted into a deck.
    (The second layout spans 88 columns; a deck reader that keeps 80 of them,
    as MCM's does, loses the energy's exponent.)"""
    x, disp, mat = state["x"], state["dispbc"], state["mat"]
    out = ["*\n* Node Coordinates and Materials\n*\n"]
    out.extend(f"{i + 1:8d}{int(disp[i]):5d}" + "".join(fmt_e(c, 20, 13) for c in x[i]) + f"{int(mat[i]):7d}\n"
               for i in range(x.shape[0]))
    out.append("*\n* Node Data\n*     ID  Mass                Smoothing Length    Density             Internal Energy\n")
    cols = np.stack([state["mass"], state["h"], state["rho"], state["e"]], axis=1)
    out.extend(f"{i + 1:8d}" + "".join(fmt_e(c, 20, 13) for c in cols[i]) + "\n" for i in range(x.shape[0]))
    return "".join(out)


def state_line(ptime: float) -> str:
    """Format 1200 of MCM/mcm_solution.f90:145, printed after each state output."""
    return f"\n     State plot written at time {fmt_e(ptime, 10, 4)}"


def status_line(timestep: int, ptime: float, dt: float) -> str:
    """Format 1000 of MCM/mcm_solution.f90:143-144."""
    return (f"\n     Problem status for time-step {fmt_i(timestep, 6)}\n"
            f"     Time: {fmt_e(ptime, 10, 4)}     dt: {fmt_e(dt, 10, 4)}")
