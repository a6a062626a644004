"""Host loop mirroring MCM/mcm_solution.f90, driving the GPU step through the
C ABI of libmcm_gpu.so (include/mcm_gpu.h).

:class:`Solver` owns one device handle.  ``step()`` runs one iteration of the
reference loop through the split entry points (step_a / host dt update /
step_b / termination test / step_c), exactly where the Fortran driver would
call them; ``run(n)`` runs n iterations with the dt update and termination
test on the device.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import check
from .deck import Deck

_SYM_FIELDS = ("sigma", "s", "q", "qold", "alfa", "rod", "spin")


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def material_table(deck: Deck) -> "C.Array":
    """Material structures after the deck defaults and mcm_sets* (done by the library)."""
    lib = _abi.load()
    n = len(deck.materials)
    mats = (_abi.Material * n)()
    for k, card in enumerate(deck.materials):
        m = mats[k]
        m.model, m.eos, m.visc_type = card.model, card.eos, card.visc_type
        m.rho, m.av_l, m.av_q, m.mass, m.h = card.rho, card.av_l, card.av_q, card.mass, card.h
        m.rho_min, m.rho_max = card.rho_min, card.rho_max
        for i in range(48):
            m.strinput[i] = float(card.strinput[i])
        for i in range(24):
            m.eosinput[i] = float(card.eosinput[i])
        check(lib.mcm_gpu_material_from_deck(C.byref(m)), "mcm_gpu_material_from_deck")
        # contact cards (MCM/mcm_contactype.f90:32-39): K and n per material
        if deck.contacttype > 0 and k < len(deck.k_cont):
            m.k_cont, m.n_cont = float(deck.k_cont[k]), float(deck.n_cont[k])
    return mats


def config_from_deck(deck: Deck, precision: int, nbr_stride: int = 0, reorder_interval: int = 0,
                     nbr_skin: float = 0.0, compensated: bool = False) -> _abi.Config:
    """Control-card processing of MCM/mcm_control_v2.f90:193-243 and the
    boundary/base-acceleration cards (mcm_inp_symmetry_v2.f90:83-137,
    mcm_baseaccel_in.f90:23-33)."""
    c = _abi.Config()
    c.ndim = deck.ndim
    c.disctype = deck.disctype
    c.tcrit_opt = deck.tcrit_opt
    c.contacttype = deck.contacttype
    c.h_opt = deck.h_opt
    c.veloc_opt = deck.veloc_opt
    c.krtype = deck.krtype if deck.krtype else 1
    c.drelax = int(0.1 < deck.drelax_scale < 1.0)
    c.drelax_scale = deck.drelax_scale
    boundary = deck.mirr_opt == 1 and any(f in (1, 2) for f in deck.sym_flag)
    c.boundary = int(boundary)
    for k in range(6):
        c.boundary_code[k] = int(deck.sym_flag[k]) if boundary else 0
        c.boundary_x[k] = float(deck.sym_x[k])
    c.baseaccel = int(any(t == 1 for t in deck.nthp))
    for k in range(3):
        c.base_a[k] = float(deck.base_a[k]) if deck.nthp[k] == 1 else 0.0
    c.tssf = deck.tssf if deck.tssf != 0.0 else 0.8
    c.hmax = 0.0
    c.precision = precision
    c.nbr_stride = nbr_stride
    c.reorder_interval = reorder_interval
    c.nbr_skin = nbr_skin
    c.compensated_sums = int(bool(compensated))
    return c


class Solver:
    def __init__(self, deck: Deck, precision: int = _abi.PREC_FP64_EXACT, nbr_stride: int = 0,
                 device: int | None = None, reorder_interval: int = 0, nbr_skin: float = 0.0,
                 compensated: bool = False):
        self.lib = _abi.load()
        if device is not None:
            check(self.lib.mcm_gpu_set_device(int(device)), "mcm_gpu_set_device")
        self.deck = deck
        self.n = deck.np
        self.nmat = len(deck.materials)
        self._mats = material_table(deck)
        self.cfg = config_from_deck(deck, precision, nbr_stride, reorder_interval, nbr_skin, compensated)
        h = C.c_void_p()
        check(self.lib.mcm_gpu_create(C.byref(self.cfg), self._mats, self.nmat, self.n, C.byref(h)),
              "mcm_gpu_create")
        self.h = h
        x = np.ascontiguousarray(deck.x, dtype=np.float64)
        v = np.ascontiguousarray(deck.v if deck.init_v_opt == 1 else np.zeros_like(deck.x), dtype=np.float64)
        mat = np.ascontiguousarray(deck.mat, dtype=np.int32)
        disp = np.ascontiguousarray(deck.dispbc if deck.dispbc is not None else np.zeros(self.n), dtype=np.int32)
        f = _abi.Fields()
        f.x, f.v, f.mat, f.dispbc = _dptr(x), _dptr(v), _iptr(mat), _iptr(disp)
        keep = []
        if deck.pardata is not None:
            # additional particle cards (MCM/mcm_nodein.f90:76-112): mass, h, rho, e
            for col, nm in enumerate(("mass", "h", "rho", "e")):
                a = np.ascontiguousarray(np.asarray(deck.pardata, dtype=np.float64)[:, col])
                keep.append(a)
                setattr(f, nm, _dptr(a))
        t = _abi.Time(0.0, 0.0, 0.0, deck.endtime)
        check(self.lib.mcm_gpu_initialise(h, C.byref(f), deck.massopt, deck.init_h_opt, deck.init_rhoe,
                                          deck.itss, C.byref(t)), "mcm_gpu_initialise", h)
        self.dt, self.dtold, self.ptime = t.dt, t.dtold, t.ptime
        self.tssf = self.cfg.tssf
        self.timestep = 1
        self.ended = False
        self.energies = np.zeros(5 * self.nmat + 3)
        self.bbox = np.zeros(6)
        self.last_critts = None

    # ------------------------------------------------------------- loop
    def step_a(self) -> float:
        crit = C.c_double()
        check(self.lib.mcm_gpu_step_a(self.h, self.dt, C.byref(crit)), "mcm_gpu_step_a", self.h)
        self.last_critts = crit.value
        return crit.value

    def dt_update(self) -> None:
        # MCM/mcm_solution.f90:58-62
        self.dtold = self.dt
        self.dt = self.tssf * self.last_critts
        self.dt = min(self.dt, 1.1 * self.dtold)
        self.ptime = self.ptime + self.dt

    def step_b(self, energies: bool = True):
        """mcm_gpu_step_b; with energies False it only enqueues the step's work
        (a driver that reads the energies at output times, energies_now())."""
        if not energies:
            check(self.lib.mcm_gpu_step_b(self.h, None), "mcm_gpu_step_b", self.h)
            return None
        check(self.lib.mcm_gpu_step_b(self.h, _dptr(self.energies)), "mcm_gpu_step_b", self.h)
        return self.energies

    def energies_now(self) -> np.ndarray:
        """The energies of the last mcm_calctotale (step_b or initialisation)."""
        e = np.zeros(5 * self.nmat + 3)
        check(self.lib.mcm_gpu_energies(self.h, _dptr(e)), "mcm_gpu_energies", self.h)
        return e

    def step_c(self, bbox: bool = False) -> None:
        """Velocity and position update; bbox=True also reads mcm_coord_maxmin
        into self.bbox (a wait), otherwise the call returns without waiting."""
        check(self.lib.mcm_gpu_step_c(self.h, self.dt, self.dtold, _dptr(self.bbox) if bbox else None),
              "mcm_gpu_step_c", self.h)
        self.timestep += 1

    def step(self, energies: bool = True) -> bool:
        """One iteration of MCM/mcm_solution.f90:37-138; False once it terminates.
        energies False: step_b does not wait for the energy sums."""
        if self.ended:
            return False
        self.step_a()
        self.dt_update()
        self.step_b(energies)
        if self.ptime - self.dt >= self.deck.endtime:   # :101
            self.ended = True
            return False
        self.step_c()
        return True

    def run(self, nsteps: int) -> int:
        """nsteps iterations with the time scalars kept on the device."""
        t = _abi.Time(self.dt, self.dtold, self.ptime, self.deck.endtime)
        done = C.c_int()
        check(self.lib.mcm_gpu_run(self.h, nsteps, C.byref(t), C.byref(done)), "mcm_gpu_run", self.h)
        self.dt, self.dtold, self.ptime = t.dt, t.dtold, t.ptime
        self.timestep += done.value
        if done.value < nsteps or self.ptime - self.dt >= self.deck.endtime:
            self.ended = self.ptime - self.dt >= self.deck.endtime
        return done.value

    # ------------------------------------------------------- inspection
    def download_into(self, buffers: dict) -> None:
        """mcm_gpu_download into the caller's buffers in the ABI's layout
        (C-contiguous: vectors (np, 3) = Fortran (3,np), tensors (np, 3, 3)
        holding Fortran (3,3,np) column-major records, ints int32), e.g.
        page-locked arrays that the copies fill at the link's speed."""
        f = _abi.Fields()
        for nm, a in buffers.items():
            want = np.int32 if nm in _abi.INT_FIELDS else np.float64
            if a.dtype != want or not a.flags.c_contiguous or a.size != self.n * _abi.FIELD_WIDTH.get(nm, 1):
                raise ValueError(f"{nm}: C-contiguous {np.dtype(want).name} of {self.n} records expected")
            setattr(f, nm, _iptr(a) if want is np.int32 else _dptr(a))
        check(self.lib.mcm_gpu_download(self.h, C.byref(f)), "mcm_gpu_download", self.h)

    def download(self, names=None) -> dict:
        if names is None:
            names = _abi.DOUBLE_FIELDS + _abi.INT_FIELDS
        f = _abi.Fields()
        out = {}
        for nm in names:
            if nm in _abi.INT_FIELDS:
                arr = np.zeros(self.n, dtype=np.int32)
                setattr(f, nm, _iptr(arr))
            else:
                w = _abi.FIELD_WIDTH.get(nm, 1)
                arr = np.zeros(self.n * w, dtype=np.float64)
                setattr(f, nm, _dptr(arr))
            out[nm] = arr
        check(self.lib.mcm_gpu_download(self.h, C.byref(f)), "mcm_gpu_download", self.h)
        for nm, arr in out.items():
            w = _abi.FIELD_WIDTH.get(nm, 1)
            if w == 3:
                out[nm] = arr.reshape(self.n, 3)
            elif w == 9:
                # Fortran (3,3): element (r,c) at r + 3c -> [i, r, c]
                out[nm] = arr.reshape(self.n, 3, 3).transpose(0, 2, 1)
        return out

    def neighbours(self):
        """(nnbr, nbr[np, stride], g_nnbr, g_nbr[np, g_stride]) with 1-based ids."""
        nn = np.zeros(self.n, dtype=np.int32)
        gn = np.zeros(self.n, dtype=np.int32)
        s, gs = C.c_int(0), C.c_int(0)
        check(self.lib.mcm_gpu_neighbours(self.h, _iptr(nn), None, C.byref(s), _iptr(gn), None, C.byref(gs)),
              "mcm_gpu_neighbours", self.h)
        stride, gstride = max(1, s.value), max(1, gs.value)
        nbr = np.zeros((self.n, stride), dtype=np.int32)
        gnbr = np.zeros((self.n, gstride), dtype=np.int32)
        s, gs = C.c_int(stride), C.c_int(gstride)
        check(self.lib.mcm_gpu_neighbours(self.h, _iptr(nn), _iptr(nbr), C.byref(s), _iptr(gn), _iptr(gnbr),
                                          C.byref(gs)), "mcm_gpu_neighbours", self.h)
        return nn, nbr, gn, gnbr

    def skin_builds(self) -> int:
        """Skin-list builds since the handle was created (nbr_skin > 0)."""
        n = C.c_longlong()
        check(self.lib.mcm_gpu_skin_builds(self.h, C.byref(n)), "mcm_gpu_skin_builds", self.h)
        return n.value

    def contacts(self):
        """(ncont, cont[np, stride], g_ncont, g_cont[np, g_stride]) with 1-based ids:
        the contact lists of the last search (contacttype > 0)."""
        nc = np.zeros(self.n, dtype=np.int32)
        gc = np.zeros(self.n, dtype=np.int32)
        s, gs = C.c_int(0), C.c_int(0)
        check(self.lib.mcm_gpu_contacts(self.h, _iptr(nc), None, C.byref(s), _iptr(gc), None, C.byref(gs)),
              "mcm_gpu_contacts", self.h)
        stride, gstride = max(1, s.value), max(1, gs.value)
        cont = np.zeros((self.n, stride), dtype=np.int32)
        gcont = np.zeros((self.n, gstride), dtype=np.int32)
        s, gs = C.c_int(stride), C.c_int(gstride)
        check(self.lib.mcm_gpu_contacts(self.h, _iptr(nc), _iptr(cont), C.byref(s), _iptr(gc), _iptr(gcont),
                                        C.byref(gs)), "mcm_gpu_contacts", self.h)
        return nc, cont, gc, gcont

    def contact_forces(self) -> np.ndarray:
        """Per-material contact forces (xcf, ycf, zcf) of the last step_b, shape (nmat, 3)."""
        out = np.zeros(3 * self.nmat)
        check(self.lib.mcm_gpu_contact_forces(self.h, _dptr(out)), "mcm_gpu_contact_forces", self.h)
        return out.reshape(self.nmat, 3)

    def ghosts(self):
        n = C.c_int()
        check(self.lib.mcm_gpu_ghosts(self.h, C.byref(n), None, None, None, 0), "mcm_gpu_ghosts", self.h)
        m = n.value
        par = np.zeros(max(m, 1), dtype=np.int32)
        x = np.zeros(max(m, 1) * 3)
        v = np.zeros(max(m, 1) * 3)
        check(self.lib.mcm_gpu_ghosts(self.h, C.byref(n), _iptr(par), _dptr(x), _dptr(v), m), "mcm_gpu_ghosts", self.h)
        return par[:m], x[: 3 * m].reshape(m, 3), v[: 3 * m].reshape(m, 3)

    def grid(self):
        gl = np.zeros(3, dtype=np.int32)
        gm = np.zeros(3)
        gs = np.zeros(3)
        check(self.lib.mcm_gpu_grid(self.h, _iptr(gl), _dptr(gm), _dptr(gs)), "mcm_gpu_grid", self.h)
        return gl, gm, gs

    def stats(self):
        mean = C.c_double()
        mx, st, ngp = C.c_int(), C.c_int(), C.c_int()
        check(self.lib.mcm_gpu_stats(self.h, C.byref(mean), C.byref(mx), C.byref(st), C.byref(ngp)), "mcm_gpu_stats",
              self.h)
        return {"mean_nbr": mean.value, "max_nbr": mx.value, "stride": st.value, "ngp": ngp.value}

    # ---------------------------------------------------------- adjoint
    def adjoint_forward(self, dts, checkpoint_every: int = 50) -> None:
        """Runs len(dts) - 1 steps with the prescribed dt schedule, keeping
        checkpoints for adjoint_backward (mcm_gpu_adjoint_forward)."""
        d = np.ascontiguousarray(dts, dtype=np.float64)
        check(self.lib.mcm_gpu_adjoint_forward(self.h, len(d) - 1, _dptr(d), int(checkpoint_every)),
              "mcm_gpu_adjoint_forward", self.h)
        self.dtold, self.dt = float(d[-2]), float(d[-1])

    def adjoint_backward(self, xbar=None, vbar=None):
        """Adjoints of the final x, v ((np, 3) arrays) -> (param_bar (nmat, 4):
        d/d(G, yield, hardening, EOS-41 s) in card units, xbar0, vbar0)."""
        keep = []

        def arg(a):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(a)
            return _dptr(a)

        pb = np.zeros((self.nmat, 4))
        x0 = np.zeros((self.n, 3))
        v0 = np.zeros((self.n, 3))
        check(self.lib.mcm_gpu_adjoint_backward(self.h, arg(xbar), arg(vbar), _dptr(pb), _dptr(x0), _dptr(v0)),
              "mcm_gpu_adjoint_backward", self.h)
        return pb, x0, v0

    # ------------------------------------------------------ launch shape
    def tuning(self) -> dict:
        t = _abi.Tuning()
        check(self.lib.mcm_gpu_get_tuning(self.h, C.byref(t)), "mcm_gpu_get_tuning", self.h)
        return {k: getattr(t, k) for k, _ in _abi.Tuning._fields_}

    def set_tuning(self, search_threads: int = 0, pair_threads: int = 0, pair_blocks_per_sm: int = 0,
                   nbr_stride: int = 0, search_kind: int = 0, pair_kind: int = 0, adj_kind: int = 0) -> None:
        """search_kind 1: one thread per particle, 2: one warp per particle, 3: one warp per cell;
        pair_kind (mixed gathers) 1: records through L1, 2: rows staged in shared memory;
        adj_kind (reverse constitutive step) 1: hand-written reverse for model 10 + EOS 41, 2: dual numbers."""
        t = _abi.Tuning(search_threads, pair_threads, pair_blocks_per_sm, nbr_stride, search_kind, pair_kind,
                        adj_kind, 0.0)
        check(self.lib.mcm_gpu_set_tuning(self.h, C.byref(t)), "mcm_gpu_set_tuning", self.h)

    def autotune(self, nsteps: int = 5) -> dict:
        """Times candidate launch shapes over nsteps iterations from the
        current state (which is restored) and keeps the fastest."""
        t = _abi.Tuning()
        check(self.lib.mcm_gpu_autotune(self.h, int(nsteps), C.byref(t)), "mcm_gpu_autotune", self.h)
        return {k: getattr(t, k) for k, _ in _abi.Tuning._fields_}

    # ------------------------------------------------------ measurement
    def set_diagnostics(self, enable: bool) -> None:
        check(self.lib.mcm_gpu_set_diagnostics(self.h, int(enable)), "mcm_gpu_set_diagnostics", self.h)

    def profile(self, enable: bool) -> None:
        check(self.lib.mcm_gpu_profile(self.h, int(enable)), "mcm_gpu_profile", self.h)

    def profile_report(self) -> dict:
        """{kernel group: (total device ms, launches)} since profile(True)."""
        out = {}
        r = 0
        buf = C.create_string_buffer(64)
        while True:
            ms, n = C.c_double(), C.c_int()
            st = self.lib.mcm_gpu_profile_report(self.h, r, buf, 64, C.byref(ms), C.byref(n))
            if st == _abi.MCM_EINVAL:
                break
            check(st, "mcm_gpu_profile_report", self.h)
            out[buf.value.decode()] = (ms.value, n.value)
            r += 1
        return out

    def kernel_launches(self) -> int:
        return int(self.lib.mcm_gpu_kernel_launches(self.h))

    def timer_start(self) -> None:
        check(self.lib.mcm_gpu_timer(self.h, 0, None), "mcm_gpu_timer", self.h)

    def timer_stop(self) -> float:
        ms = C.c_double()
        check(self.lib.mcm_gpu_timer(self.h, 1, C.byref(ms)), "mcm_gpu_timer", self.h)
        return ms.value

    def upload(self, state: dict, bbox=None, fortran_layout: bool = False) -> None:
        """Uploads a host state (the fields a Fortran driver passes) through
        mcm_gpu_upload.  Arrays are [particle, ...] as download returns them;
        with fortran_layout=True they are already the ABI's buffers (vectors
        (3,np), tensors (3,3,np) column-major, C-contiguous float64/int32) and
        are passed as they are, without a host copy."""
        f = _abi.Fields()
        keep = []
        for nm, arr in state.items():
            if nm in _abi.INT_FIELDS:
                a = arr if fortran_layout else np.ascontiguousarray(arr, dtype=np.int32)
                if a.dtype != np.int32 or not a.flags.c_contiguous:
                    raise ValueError(f"{nm}: C-contiguous int32 expected")
                setattr(f, nm, _iptr(a))
            else:
                if fortran_layout:
                    a = arr
                    if a.dtype != np.float64 or not a.flags.c_contiguous:
                        raise ValueError(f"{nm}: C-contiguous float64 expected")
                else:
                    a = np.asarray(arr, dtype=np.float64)
                    if a.ndim == 3:
                        a = a.transpose(0, 2, 1)
                    a = np.ascontiguousarray(a)
                setattr(f, nm, _dptr(a))
            if a.size != self.n * _abi.FIELD_WIDTH.get(nm, 1):
                raise ValueError(f"{nm}: {self.n} records of {_abi.FIELD_WIDTH.get(nm, 1)} expected, got {a.size} values")
            keep.append(a)
        b = None
        if bbox is not None:
            b = np.ascontiguousarray(bbox, dtype=np.float64)
            if b.size != 6:
                raise ValueError("bbox: xmin xmax ymin ymax zmin zmax expected")
            keep.append(b)
        check(self.lib.mcm_gpu_upload(self.h, C.byref(f), _dptr(b) if b is not None else None), "mcm_gpu_upload",
              self.h)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.mcm_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent bodies advanced together (mcm_gpu_batch_*): one loop
    iteration of every body per CUDA-graph launch, bodies spread over `lanes`
    streams.  The solvers keep their own time scalars; run() updates them."""

    def __init__(self, solvers, lanes: int = 8):
        self.lib = _abi.load()
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(self.solvers))(*[s.h.value for s in self.solvers])
        b = C.c_void_p()
        check(self.lib.mcm_gpu_batch_create(arr, len(self.solvers), int(lanes), C.byref(b)), "mcm_gpu_batch_create",
              self.solvers[0].h)
        self.b = b

    def _times(self):
        return (_abi.Time * len(self.solvers))(*[_abi.Time(s.dt, s.dtold, s.ptime, s.deck.endtime)
                                                  for s in self.solvers])

    def adjoint_forward(self, dts_per_body, checkpoint_every: int = 50) -> None:
        """mcm_gpu_adjoint_forward of every body at once (mcm_gpu_batch_adjoint_forward):
        body b runs len(dts_per_body[b]) - 1 steps with its prescribed dt schedule."""
        ds = [np.ascontiguousarray(d, dtype=np.float64) for d in dts_per_body]
        if len(ds) != len(self.solvers) or len({len(d) for d in ds}) != 1:
            raise ValueError("one dt schedule per body, all of the same length")
        ptrs = (_abi._DP * len(ds))(*[_dptr(d) for d in ds])
        check(self.lib.mcm_gpu_batch_adjoint_forward(self.b, len(ds[0]) - 1, ptrs, int(checkpoint_every)),
              "mcm_gpu_batch_adjoint_forward", self.solvers[0].h)
        for s_, d in zip(self.solvers, ds):
            s_.dtold, s_.dt = float(d[-2]), float(d[-1])

    def adjoint_backward(self, xbars=None, vbars=None):
        """mcm_gpu_batch_adjoint_backward: per body the adjoints of its final x, v
        ((np, 3) arrays or None) -> lists of (param_bar (nmat, 4), xbar0, vbar0)."""
        n = len(self.solvers)
        keep = []

        def ptrs(arrays):
            if arrays is None:
                return None
            out = []
            for a in arrays:
                a = np.ascontiguousarray(a, dtype=np.float64)
                keep.append(a)
                out.append(_dptr(a))
            return (_abi._DP * n)(*out)

        pb = [np.zeros((s_.nmat, 4)) for s_ in self.solvers]
        x0 = [np.zeros((s_.n, 3)) for s_ in self.solvers]
        v0 = [np.zeros((s_.n, 3)) for s_ in self.solvers]
        outs = [(_abi._DP * n)(*[_dptr(a) for a in arrs]) for arrs in (pb, x0, v0)]
        check(self.lib.mcm_gpu_batch_adjoint_backward(self.b, ptrs(xbars), ptrs(vbars), *outs),
              "mcm_gpu_batch_adjoint_backward", self.solvers[0].h)
        return pb, x0, v0

    def run(self, nsteps: int) -> np.ndarray:
        """nsteps iterations of every body; returns the iterations each completed."""
        t = self._times()
        done = np.zeros(len(self.solvers), dtype=np.int32)
        check(self.lib.mcm_gpu_batch_run(self.b, int(nsteps), t, _iptr(done)), "mcm_gpu_batch_run",
              self.solvers[0].h)
        for s, tk, d in zip(self.solvers, t, done):
            s.dt, s.dtold, s.ptime = tk.dt, tk.dtold, tk.ptime
            s.timestep += int(d)
            if d < nsteps or s.ptime - s.dt >= s.deck.endtime:
                s.ended = s.ptime - s.dt >= s.deck.endtime
        return done

    def autotune(self, nsteps: int = 3):
        lanes, ms = C.c_int(), C.c_double()
        check(self.lib.mcm_gpu_batch_autotune(self.b, int(nsteps), C.byref(lanes), C.byref(ms)),
              "mcm_gpu_batch_autotune", self.solvers[0].h)
        return lanes.value, ms.value

    def close(self) -> None:
        if getattr(self, "b", None):
            self.lib.mcm_gpu_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
