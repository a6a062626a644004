"""Synthetic input decks for the MCM explicit step.

A :class:`Deck` holds what MCM's version-2 input file gives the solver: the
control cards (MCM/mcm_control_v2.f90:88-124), the material cards
(MCM/mcm_matin.f90:41-148), the node cards (MCM/mcm_nodein.f90:33-43), the
initial velocities (MCM/mcm_Inputvel.f90), the boundary-plane cards
(MCM/mcm_inp_symmetry_v2.f90:29-53) and the base accelerations
(MCM/mcm_baseaccel_in.f90:27).  The reference ships no decks; the generators
below restate the benchmark configurations as seeded lattices.

Units.  The generators take SI arguments and write the deck in the DYNA3D
cm-g-microsecond system (length cm, mass g, time us, velocity cm/us, density
g/cm^3, pressure Mbar), the system MCM decks use.  The reference's Mie-
Grueneisen energy correction (MCM/mcm_eqos41.f90:81) divides by the initial
volume where the mass belongs, which multiplies the correction by the density;
with rho = 8930 in SI units its denominator changes sign after a few steps of
impact, with rho = 8.93 g/cm^3 the effect is mild.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field

import numpy as np


@dataclass
class MaterialCard:
    """One material as read from its cards (before mcm_sets*)."""

    model: int
    eos: int
    rho: float
    visc_type: int = 0
    av_l: float = 0.0
    av_q: float = 0.0
    mass: float = 0.0
    h: float = 0.0
    rho_min: float = 0.0
    rho_max: float = 0.0
    strinput: np.ndarray = field(default_factory=lambda: np.zeros(48))
    eosinput: np.ndarray = field(default_factory=lambda: np.zeros(24))
    head: str = ""           # material heading card (12a6)
    eos_head: str = ""       # EOS heading card (12a6)
    ihq: int = 0             # hourglass type and coefficient: read, not used
    qh: float = 0.0


@dataclass
class Deck:
    ndim: int = 3
    disctype: int = 0
    endtime: float = 1.0
    tssf: float = 0.8
    itss: float = 0.0
    drelax_scale: float = 0.0
    init_v_opt: int = 1
    massopt: int = 0
    init_h_opt: int = 0
    init_rhoe: int = 0
    contacttype: int = 0
    tcrit_opt: int = 0
    veloc_opt: int = 0
    mirr_opt: int = 0
    nthp: tuple = (0, 0, 0)
    h_opt: int = 0
    krtype: int = 1
    maxnbr: int = 0
    sym_flag: tuple = (0, 0, 0, 0, 0, 0)
    sym_x: tuple = (0.0, 0.0, 0.0, 0.0, 0.0, 0.0)
    base_a: tuple = (0.0, 0.0, 0.0)
    materials: list = field(default_factory=list)
    x: np.ndarray = None          # (np, 3)
    v: np.ndarray = None          # (np, 3)
    mat: np.ndarray = None        # (np,) 1-based material ids
    dispbc: np.ndarray = None     # (np,)
    name: str = "deck"
    # cards that select output and bookkeeping (MCM/mcm_control_v2.f90:92-115)
    title: str = ""
    max_np: int = 0
    nstressp: int = 0
    nvelocp: int = 0
    stpltime: float = 0.0
    state_opt: int = 0
    thpltime: float = 0.0
    status_interval: int = 0
    restart_interval: int = 0
    run_restart: int = 0
    keep_files: int = 0
    nlcur: int = 0
    thnodes: tuple = ()           # time-history particle ids (1-based)
    transducers: tuple = ()       # ((x, y, z), mat) per pressure transducer
    pardata: np.ndarray = None    # (np, 4): mass, h, rho, e when massopt/init_h_opt/init_rhoe is 1
    ncontmats: int = 0            # contact cards (MCM/mcm_contactype.f90)
    cont_opt: int = 0
    k_cont: tuple = ()
    n_cont: tuple = ()

    @property
    def np(self) -> int:
        return int(self.x.shape[0])

    def replace(self, **kw) -> "Deck":
        return dataclasses.replace(self, **kw)


def _jitter(rng: np.random.Generator, shape, amp: float) -> np.ndarray:
    return rng.uniform(-amp, amp, size=shape)


# SI -> cm-g-us conversion factors
CM = 1.0e2            # m -> cm
VEL = 1.0e-4          # m/s -> cm/us
RHO = 1.0e-3          # kg/m^3 -> g/cm^3
PRESS = 1.0e-11       # Pa -> Mbar
ACC = 1.0e-10         # m/s^2 -> cm/us^2


@dataclass(frozen=True)
class Units:
    """SI -> deck unit factors for length, velocity, density and pressure."""
    length: float
    velocity: float
    density: float
    pressure: float


CGUS = Units(CM, VEL, RHO, PRESS)          # cm, g, us: pressure in Mbar (the metal decks)
MMMSG = Units(1.0e3, 1.0, 1.0e-6, 1.0e-6)  # mm, ms, g: pressure in MPa, velocity in m/s (the soil deck)


def copper_model10(h: float, yield_stress: float = 400e6, hardening: float = 100e6, shear: float = 46e9,
                   gruneisen_s: float = 1.49, rho0: float = 8930.0) -> MaterialCard:
    """Copper-like elastic-plastic hydrodynamic material (model 10) with the
    Mie-Grueneisen EOS (41); SI arguments, cm-g-us card values; h in cm.  strinput follows MCM/mcm_f3dm10.f90:29-36
    (G, yield, plastic modulus, cutoff, a1, a2, spall, failure strain);
    eosinput follows MCM/mcm_eos41c.f90:31-36 (c0, s, cv, T0, gamma0, v0)."""
    m = MaterialCard(model=10, eos=41, rho=rho0 * RHO, av_l=0.06, av_q=1.5, h=h)
    m.strinput[0] = shear * PRESS
    m.strinput[1] = yield_stress * PRESS
    m.strinput[2] = hardening * PRESS
    m.eosinput[0] = 3940.0 * VEL
    m.eosinput[1] = gruneisen_s
    m.eosinput[2] = 0.0      # cv * T0 = 0: zero initial internal energy
    m.eosinput[3] = 0.0
    m.eosinput[4] = 2.02
    m.eosinput[5] = 1.0      # v0 = 1 (MCM/mcm_eoscalc.f90:93 divides rho0 by it)
    return m


def taylor_bar(dx: float = 0.4e-3, radius: float = 3.2e-3, length: float = 32.4e-3, velocity: float = 190.0,
               seed: int = 1234, jitter: float = 0.01, disctype: int = 0, tssf: float = 0.3,
               endtime: float = 1.0e9, material: MaterialCard | None = None, z0: float = 0.0,
               tcrit_opt: int = 1, units: Units = CGUS) -> Deck:
    """Taylor impact bar: a cylinder (axis z) of lattice particles at
    (i+1/2, j+1/2, k+1/2) dx inside r <= R, 0 < z <= L, each displaced by a
    seeded uniform jitter of +/- jitter*dx per coordinate, moving at -velocity
    along z onto a rigid wall imposed by a z-min symmetry plane at z = 0.
    Particle order: z layers, then y rows, then x.  Arguments in SI units; the
    deck is in `units` (cm-g-us by default; a given material must be in the
    same units)."""
    q = radius / dx
    n = int(np.ceil(q)) + 1
    ii = np.arange(-n, n)
    I, J = np.meshgrid(ii, ii, indexing="xy")
    inside = (2 * I + 1) ** 2 + (2 * J + 1) ** 2 <= (2.0 * q) ** 2 * (1 + 1e-12)
    dxc = dx * units.length
    xs = (I[inside] + 0.5) * dxc
    ys = (J[inside] + 0.5) * dxc
    order = np.lexsort((xs, ys))
    xs, ys = xs[order], ys[order]
    nz = int(round(length / dx))
    zs = z0 * units.length + (np.arange(nz) + 0.5) * dxc
    x = np.empty((nz * xs.size, 3))
    x[:, 0] = np.tile(xs, nz)
    x[:, 1] = np.tile(ys, nz)
    x[:, 2] = np.repeat(zs, xs.size)
    rng = np.random.default_rng(seed)
    x += _jitter(rng, x.shape, jitter * dxc)
    npart = x.shape[0]
    v = np.zeros_like(x)
    v[:, 2] = -velocity * units.velocity
    h = 1.3 * dxc
    mat = material if material is not None else copper_model10(h)
    mat = dataclasses.replace(mat, strinput=mat.strinput.copy(), eosinput=mat.eosinput.copy(), h=h)
    mat.mass = mat.rho * npart * dxc ** 3
    return Deck(ndim=3, disctype=disctype, endtime=endtime, tssf=tssf, tcrit_opt=tcrit_opt, mirr_opt=1,
                sym_flag=(0, 0, 0, 0, 1, 0), sym_x=(0.0,) * 6, materials=[mat], x=x, v=v,
                mat=np.ones(npart, dtype=np.int32), dispbc=np.zeros(npart, dtype=np.int32),
                name=f"taylor_bar_dx{dx * 1e3:g}mm_n{npart}")


def two_material_bar(dx: float = 0.8e-3, contacttype: int = 0, k_cont: float = 1.0e-3, n_cont: float = 4.0,
                     yields=(400e6, 250e6), **kw) -> Deck:
    """A Taylor bar whose lower half is material 1 and upper half material 2
    (the same copper-like model 10 + EOS 41 with the yield stresses `yields`).
    With contacttype 0 the halves are each other's neighbours (kernel
    contact); with contacttype > 0 they interact only through Monaghan's
    repulsive force, with the contact cards' strength K and exponent n for
    both materials (MCM/mcm_contactype.f90:32-39, cm-g-us units: K in
    (cm/us)^2).  Other arguments as taylor_bar."""
    d = taylor_bar(dx=dx, **kw)
    upper = d.x[:, 2] > 0.5 * (d.x[:, 2].min() + d.x[:, 2].max())
    mat = np.where(upper, 2, 1).astype(np.int32)
    dxc = dx * CM
    mats = []
    for k, ys in ((1, yields[0]), (2, yields[1])):
        m1 = d.materials[0]
        m = dataclasses.replace(m1, strinput=m1.strinput.copy(), eosinput=m1.eosinput.copy())
        m.strinput[1] = ys * PRESS
        m.mass = m.rho * int((mat == k).sum()) * dxc ** 3
        mats.append(m)
    extra = {}
    if contacttype > 0:
        extra = dict(ncontmats=-1, cont_opt=0, k_cont=(k_cont, k_cont), n_cont=(n_cont, n_cont))
    return d.replace(materials=mats, mat=mat, contacttype=contacttype,
                     name=f"two_material_bar_dx{dx * 1e3:g}mm_n{d.np}_ct{contacttype}", **extra)


def sand_model4(h: float, bulk: float = 1.0e9, shear: float = 0.6e9, alpha: float = 10e6, theta: float = 0.1,
                gamma: float = 8e6, beta: float = 0.1e-6, r: float = 2.5, d: float = 0.002e-6, w: float = 0.05,
                x0: float = 30e6, tcut: float = -1e6, rho0: float = 1800.0, iterate: bool = False,
                units: Units = MMMSG) -> MaterialCard:
    """Granular material for the cap model (model 4, MCM/mcm_f3dm25.f90):
    failure surface Fe(J1) = alpha - gamma exp(-beta J1) + theta J1, cap
    ratio R, hardening law W (1 - exp(-D (X - X0))), tension cut-off, soil
    (ltype 1).  SI arguments (Pa, 1/Pa); card values in `units`, by default
    mm-ms-g (MPa): the model's absolute tolerances (1e-3 in the initial-cap
    iteration of MCM/mcm_sets4.f90:61, 1e-7 and 1e-8 in MCM/mcm_f3dm25.f90)
    assume stresses of order 1-100, as in MPa or psi decks.  The cards
    fill the 5-row table cm(i, j) = strinput(i + 5(j-1)) as MCM/mcm_matin.f90
    reads 6 cards of 5 values: K, R, tcut, falfac | G, D | alpha, W | theta,
    X0 (hardening) | gamma, X0 (initial cap, MCM/mcm_sets4.f90:28), vector
    flag | beta, ltype.  iterate = True selects the iterated return
    (feit/fcit, cm(3,5) /= 0) instead of four fixed iterations."""
    m = MaterialCard(model=4, eos=0, rho=rho0 * units.density, av_l=0.06, av_q=1.5, h=h)
    cm = lambda i, j: (i - 1) + 5 * (j - 1)   # noqa: E731
    m.strinput[cm(1, 1)] = bulk * units.pressure
    m.strinput[cm(2, 1)] = r
    m.strinput[cm(3, 1)] = tcut * units.pressure
    m.strinput[cm(1, 2)] = shear * units.pressure
    m.strinput[cm(2, 2)] = d / units.pressure
    m.strinput[cm(1, 3)] = alpha * units.pressure
    m.strinput[cm(2, 3)] = w
    m.strinput[cm(1, 4)] = theta
    m.strinput[cm(2, 4)] = x0 * units.pressure
    m.strinput[cm(1, 5)] = gamma * units.pressure
    m.strinput[cm(2, 5)] = x0 * units.pressure
    m.strinput[cm(3, 5)] = 1.0 if iterate else 0.0
    m.strinput[cm(1, 6)] = beta / units.pressure
    m.strinput[cm(2, 6)] = 1.0
    return m


def water_model9(h: float, c0: float = 40.0, rho0: float = 1000.0, pcut: float = -1.0e4) -> MaterialCard:
    # h in cm; SI arguments otherwise
    """Null material (model 9, mu = 0) with a linear polynomial EOS (1):
    p = rho0 c0^2 mu (MCM/mcm_eqos1.f90:59-62); strinput(1) is the cutoff
    pressure (MCM/mcm_initvbls.f90:58-59)."""
    m = MaterialCard(model=9, eos=1, rho=rho0 * RHO, av_l=0.06, av_q=1.5, h=h)
    m.strinput[0] = pcut * PRESS
    m.strinput[1] = 0.0
    m.eosinput[1] = (rho0 * RHO) * (c0 * VEL) ** 2
    m.eosinput[8] = 1.0      # relative volume (MCM/mcm_eoscalc.f90:35)
    return m


def fluid_column(dx: float = 2.0e-3, block=(0.5, 0.25, 1.0), box=(2.0, 0.25, 1.2), seed: int = 4321,
                 jitter: float = 0.005, gravity: float = 9.81, tssf: float = 0.3, endtime: float = 1.0e12,
                 c0: float = 40.0) -> Deck:
    """Weakly compressible column collapse: a block of lattice particles in
    the corner of a box whose walls are symmetry planes (x-min, x-max, y-min,
    y-max, z-min), under gravity along -z (base acceleration).  Arguments in
    SI units; the deck is in cm-g-us."""
    nx, ny, nz = (int(round(b / dx)) for b in block)
    dxc = dx * CM
    gx = (np.arange(nx) + 0.5) * dxc
    gy = (np.arange(ny) + 0.5) * dxc
    gz = (np.arange(nz) + 0.5) * dxc
    Z, Y, X = np.meshgrid(gz, gy, gx, indexing="ij")
    x = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    rng = np.random.default_rng(seed)
    x += _jitter(rng, x.shape, jitter * dxc)
    npart = x.shape[0]
    h = 1.3 * dxc
    mat = water_model9(h, c0=c0)
    mat.mass = mat.rho * npart * dxc ** 3
    bx = [b * CM for b in box]
    return Deck(ndim=3, disctype=0, endtime=endtime, tssf=tssf, tcrit_opt=1, mirr_opt=1, nthp=(0, 0, 1),
                base_a=(0.0, 0.0, -gravity * ACC), sym_flag=(1, 1, 1, 1, 1, 0),
                sym_x=(0.0, bx[0], 0.0, bx[1], 0.0, bx[2]), materials=[mat], x=x,
                v=np.zeros_like(x), mat=np.ones(npart, dtype=np.int32), dispbc=np.zeros(npart, dtype=np.int32),
                name=f"fluid_column_dx{dx * 1e3:g}mm_n{npart}")


def periodic_layer(dx: float = 40e-3, size=(2.0, 0.24, 0.4), seed: int = 77, jitter: float = 0.005,
                   noise: float = 1.0, gravity: float = 9.81, tssf: float = 0.3, endtime: float = 1.0e12,
                   c0: float = 40.0) -> Deck:
    """A water layer filling a box that is periodic in x and y
    (MCM/mcm_inp_symmetry_v2.f90 flag 2 on both sides) on a z-min symmetry
    floor, under gravity, with a seeded random velocity of amplitude `noise`
    (m/s) so that particles cross the periodic planes.  SI arguments; the deck
    is in cm-g-us."""
    d = fluid_column(dx=dx, block=size, box=(size[0], size[1], 3.0 * size[2]), seed=seed, jitter=jitter,
                     gravity=gravity, tssf=tssf, endtime=endtime, c0=c0)
    rng = np.random.default_rng(seed + 1)
    v = rng.uniform(-noise, noise, size=d.x.shape) * VEL
    bx = [b * CM for b in size]
    return d.replace(v=v, sym_flag=(2, 2, 2, 2, 1, 0), sym_x=(0.0, bx[0], 0.0, bx[1], 0.0, 3.0 * bx[2]),
                     name=f"periodic_layer_dx{dx * 1e3:g}mm_n{d.np}")


def taylor_ensemble(nbodies: int = 256, seed: int = 2024, nmin: int = 4000, nmax: int = 64000,
                    radius=(2.0e-3, 4.0e-3), aspect=(6.0, 12.0), yield_stress=(200e6, 600e6),
                    velocity=(120.0, 250.0), tcrit_opt: int = 1) -> list:
    """A calibration ensemble of independent Taylor bars: radius uniform in
    `radius`, length/diameter uniform in `aspect`, particle count log-uniform
    in [nmin, nmax] (the spacing dx = (pi R^2 L / N)^(1/3) that gives it),
    yield stress and impact velocity uniform in their ranges; everything else
    as taylor_bar.  SI arguments; one seeded generator for the whole set."""
    rng = np.random.default_rng(seed)
    decks = []
    for b in range(nbodies):
        r = rng.uniform(*radius)
        length = 2.0 * r * rng.uniform(*aspect)
        n = np.exp(rng.uniform(np.log(nmin), np.log(nmax)))
        dx = (np.pi * r * r * length / n) ** (1.0 / 3.0)
        ys = rng.uniform(*yield_stress)
        v = rng.uniform(*velocity)
        mat = copper_model10(1.3 * dx * CM, yield_stress=ys)
        d = taylor_bar(dx=dx, radius=r, length=length, velocity=v, seed=seed + 1 + b, material=mat,
                       tcrit_opt=tcrit_opt)
        decks.append(d.replace(name=f"ensemble{b}_{d.name}"))
    return decks
