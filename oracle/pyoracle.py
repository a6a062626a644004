"""ctypes wrapper of the oracle (oracle/mcm_oracle.cpp): TEST INFRASTRUCTURE ONLY.

Builds the oracle's deck structures from a mcmtop_b200 Deck and exposes the
loop body split exactly like the GPU C ABI.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


class OMaterial(C.Structure):
    _fields_ = [
        ("model", C.c_int), ("eos", C.c_int), ("visc_type", C.c_int),
        ("rho", C.c_double), ("av_l", C.c_double), ("av_q", C.c_double), ("mass", C.c_double),
        ("h", C.c_double), ("rho_min", C.c_double), ("rho_max", C.c_double),
        ("strinput", C.c_double * 48), ("eosinput", C.c_double * 24),
        ("k_cont", C.c_double), ("n_cont", C.c_double),
    ]


class ODeck(C.Structure):
    _fields_ = [
        ("ndim", C.c_int), ("disctype", C.c_int), ("nummat", C.c_int), ("np", C.c_int),
        ("endtime", C.c_double), ("tssf", C.c_double), ("itss", C.c_double), ("drelax_scale", C.c_double),
        ("init_v_opt", C.c_int), ("massopt", C.c_int), ("init_h_opt", C.c_int), ("init_rhoe", C.c_int),
        ("contacttype", C.c_int), ("tcrit_opt", C.c_int), ("veloc_opt", C.c_int), ("mirr_opt", C.c_int),
        ("nthp", C.c_int * 3), ("h_opt", C.c_int), ("krtype", C.c_int), ("maxnbr", C.c_int),
        ("sym_flag", C.c_int * 6), ("sym_x", C.c_double * 6), ("base_a", C.c_double * 3),
    ]


_libs = {}


def build() -> None:
    r = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)


def load(openmp: bool = False) -> C.CDLL:
    name = "libmcm_oracle_omp.so" if openmp else "libmcm_oracle.so"
    if name in _libs:
        return _libs[name]
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    V = C.c_void_p
    DP, IP = C.POINTER(C.c_double), C.POINTER(C.c_int)
    sig = {
        "mcmo_create": ([C.POINTER(ODeck), C.POINTER(OMaterial), DP, DP, IP, IP, DP, IP], V),
        "mcmo_destroy": ([V], None),
        "mcmo_step_a": ([V, DP], C.c_int),
        "mcmo_dt_update": ([V], C.c_int),
        "mcmo_step_b": ([V], C.c_int),
        "mcmo_ended": ([V], C.c_int),
        "mcmo_step_c": ([V], C.c_int),
        "mcmo_run": ([V, C.c_int, IP], C.c_int),
        "mcmo_get": ([V, C.c_char_p, DP], C.c_int),
        "mcmo_get_int": ([V, C.c_char_p, IP], C.c_int),
        "mcmo_set": ([V, C.c_char_p, DP], C.c_int),
        "mcmo_scalar": ([V, C.c_char_p], C.c_double),
        "mcmo_set_scalar": ([V, C.c_char_p, C.c_double], C.c_int),
        "mcmo_nbrlist": ([V, C.c_int, IP, C.c_int], C.c_int),
        "mcmo_g_nbrlist": ([V, C.c_int, IP, C.c_int], C.c_int),
        "mcmo_contlist": ([V, C.c_int, IP, C.c_int], C.c_int),
        "mcmo_g_contlist": ([V, C.c_int, IP, C.c_int], C.c_int),
        "mcmo_contact_forces": ([V, DP], C.c_int),
        "mcmo_ghosts": ([V, IP, DP, DP, C.c_int], C.c_int),
        "mcmo_grid": ([V, IP, DP, DP], C.c_int),
        "mcmo_material_energy": ([V, DP, DP, DP], C.c_int),
        "mcmo_material_table": ([V, C.c_int, DP, DP, DP], C.c_int),
        "mcmo_kernel_w": ([C.c_int, DP, DP, C.c_double], C.c_double),
        "mcmo_gradw": ([C.c_int, DP, DP, C.c_double, DP], None),
    }
    for nm, (a, r) in sig.items():
        fn = getattr(lib, nm)
        fn.argtypes = a
        fn.restype = r
    _libs[name] = lib
    return lib


WIDTH = {"x": 3, "xzero": 3, "v": 3, "a": 3, "repulsion": 3, "rod": 9, "spin": 9, "sigma": 9, "s": 9, "q": 9, "qold": 9, "alfa": 9}


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class Oracle:
    """One oracle simulation initialised by its own restatement of mcm_initial."""

    def __init__(self, deck, openmp: bool = False):
        self.lib = load(openmp)
        d = ODeck()
        d.ndim, d.disctype, d.nummat, d.np = deck.ndim, deck.disctype, len(deck.materials), deck.np
        d.endtime, d.tssf, d.itss, d.drelax_scale = deck.endtime, deck.tssf, deck.itss, deck.drelax_scale
        d.init_v_opt, d.massopt, d.init_h_opt, d.init_rhoe = deck.init_v_opt, deck.massopt, deck.init_h_opt, deck.init_rhoe
        d.contacttype, d.tcrit_opt, d.veloc_opt, d.mirr_opt = deck.contacttype, deck.tcrit_opt, deck.veloc_opt, deck.mirr_opt
        for k in range(3):
            d.nthp[k] = int(deck.nthp[k])
            d.base_a[k] = float(deck.base_a[k])
        d.h_opt, d.krtype, d.maxnbr = deck.h_opt, deck.krtype, deck.maxnbr
        for k in range(6):
            d.sym_flag[k] = int(deck.sym_flag[k])
            d.sym_x[k] = float(deck.sym_x[k])
        mats = (OMaterial * len(deck.materials))()
        for k, c in enumerate(deck.materials):
            m = mats[k]
            m.model, m.eos, m.visc_type = c.model, c.eos, c.visc_type
            m.rho, m.av_l, m.av_q, m.mass, m.h = c.rho, c.av_l, c.av_q, c.mass, c.h
            m.rho_min, m.rho_max = c.rho_min, c.rho_max
            for i in range(48):
                m.strinput[i] = float(c.strinput[i])
            for i in range(24):
                m.eosinput[i] = float(c.eosinput[i])
            if deck.contacttype > 0 and k < len(deck.k_cont):
                m.k_cont, m.n_cont = float(deck.k_cont[k]), float(deck.n_cont[k])
        self.n = deck.np
        self.nmat = len(deck.materials)
        x = np.ascontiguousarray(deck.x, dtype=np.float64)
        v = np.ascontiguousarray(deck.v, dtype=np.float64)
        mat = np.ascontiguousarray(deck.mat, dtype=np.int32)
        disp = np.ascontiguousarray(deck.dispbc, dtype=np.int32)
        st = C.c_int()
        pd = None
        if getattr(deck, "pardata", None) is not None:
            pd = np.ascontiguousarray(deck.pardata, dtype=np.float64)
        self.sim = self.lib.mcmo_create(C.byref(d), mats, _dp(x), _dp(v), _ip(mat), _ip(disp),
                                        _dp(pd) if pd is not None else None, C.byref(st))
        if not self.sim:
            raise RuntimeError(f"oracle create failed: status {st.value}")

    def close(self):
        if self.sim:
            self.lib.mcmo_destroy(self.sim)
            self.sim = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step_a(self) -> float:
        c = C.c_double()
        st = self.lib.mcmo_step_a(self.sim, C.byref(c))
        if st:
            raise RuntimeError(f"oracle step_a status {st}")
        return c.value

    def dt_update(self):
        self.lib.mcmo_dt_update(self.sim)

    def step_b(self):
        self.lib.mcmo_step_b(self.sim)

    def ended(self) -> bool:
        return bool(self.lib.mcmo_ended(self.sim))

    def step_c(self):
        self.lib.mcmo_step_c(self.sim)

    def step(self) -> bool:
        self.step_a()
        self.dt_update()
        self.step_b()
        if self.ended():
            return False
        self.step_c()
        return True

    def run(self, n: int) -> int:
        done = C.c_int()
        st = self.lib.mcmo_run(self.sim, n, C.byref(done))
        if st:
            raise RuntimeError(f"oracle run status {st}")
        return done.value

    def get(self, name: str) -> np.ndarray:
        w = WIDTH.get(name, 1)
        out = np.zeros(self.n * w)
        if self.lib.mcmo_get(self.sim, name.encode(), _dp(out)):
            raise KeyError(name)
        if w == 3:
            return out.reshape(self.n, 3)
        if w == 9:
            return out.reshape(self.n, 3, 3).transpose(0, 2, 1)
        return out

    def set(self, name: str, values: np.ndarray) -> None:
        w = WIDTH.get(name, 1)
        if w == 9:
            values = np.ascontiguousarray(np.asarray(values).transpose(0, 2, 1))
        arr = np.ascontiguousarray(values, dtype=np.float64).ravel()
        if self.lib.mcmo_set(self.sim, name.encode(), _dp(arr)):
            raise KeyError(name)

    def get_int(self, name: str) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.int32)
        if self.lib.mcmo_get_int(self.sim, name.encode(), _ip(out)):
            raise KeyError(name)
        return out

    def scalar(self, name: str) -> float:
        return self.lib.mcmo_scalar(self.sim, name.encode())

    def set_scalar(self, name: str, value: float) -> None:
        self.lib.mcmo_set_scalar(self.sim, name.encode(), float(value))

    def nbrlist(self, i: int) -> np.ndarray:
        buf = np.zeros(1024, dtype=np.int32)
        n = self.lib.mcmo_nbrlist(self.sim, i, _ip(buf), 1024)
        return buf[:n].copy()

    def g_nbrlist(self, i: int) -> np.ndarray:
        buf = np.zeros(1024, dtype=np.int32)
        n = self.lib.mcmo_g_nbrlist(self.sim, i, _ip(buf), 1024)
        return buf[:n].copy()

    def contlist(self, i: int) -> np.ndarray:
        buf = np.zeros(1024, dtype=np.int32)
        n = self.lib.mcmo_contlist(self.sim, i, _ip(buf), 1024)
        return buf[:n].copy()

    def g_contlist(self, i: int) -> np.ndarray:
        buf = np.zeros(1024, dtype=np.int32)
        n = self.lib.mcmo_g_contlist(self.sim, i, _ip(buf), 1024)
        return buf[:n].copy()

    def contact_forces(self) -> np.ndarray:
        """Per material xcf, ycf, zcf of the last momentum sum, shape (nmat, 3)."""
        out = np.zeros(3 * self.nmat)
        self.lib.mcmo_contact_forces(self.sim, _dp(out))
        return out.reshape(self.nmat, 3)

    def ghosts(self):
        n = self.lib.mcmo_ghosts(self.sim, None, None, None, 0)
        par = np.zeros(max(n, 1), dtype=np.int32)
        x = np.zeros(3 * max(n, 1))
        v = np.zeros(3 * max(n, 1))
        self.lib.mcmo_ghosts(self.sim, _ip(par), _dp(x), _dp(v), n)
        return par[:n], x[: 3 * n].reshape(n, 3), v[: 3 * n].reshape(n, 3)

    def grid(self):
        gl = np.zeros(3, dtype=np.int32)
        gm = np.zeros(3)
        gs = np.zeros(3)
        self.lib.mcmo_grid(self.sim, _ip(gl), _dp(gm), _dp(gs))
        return gl, gm, gs

    def energies(self):
        ke = np.zeros(self.nmat)
        ie = np.zeros(self.nmat)
        mom = np.zeros(3 * self.nmat)
        self.lib.mcmo_material_energy(self.sim, _dp(ke), _dp(ie), _dp(mom))
        out = []
        for m in range(self.nmat):
            out += [ke[m], ie[m], mom[3 * m], mom[3 * m + 1], mom[3 * m + 2]]
        out += [self.scalar("kinetice"), self.scalar("internale"), self.scalar("totale")]
        return np.array(out)

    def material_table(self, m: int):
        si = np.zeros(48)
        ei = np.zeros(24)
        g = C.c_double()
        self.lib.mcmo_material_table(self.sim, m, _dp(si), _dp(ei), C.byref(g))
        return si, ei, g.value
