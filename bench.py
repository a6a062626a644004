"""Benchmark of the MCM explicit SPH step on B200.

Workload: the 2 034 720-particle Taylor bar (dx = 0.08 mm, copper, model 10 +
EOS 41, z-min symmetry wall), the configuration the headline metric is quoted
on.  One "step" is one iteration of MCM's time loop (neighbour search, strain,
constitutive update, dt, momentum, boundary conditions, energies, velocity and
position update) over every particle.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|exact|mixed]
  python bench.py --impl reference ...   # the CPU restatement on the host cores

value: particle-steps/s of the fused device loop (mcm_gpu_run) in the
headline precision (mixed: FP32 pair sums, FP64 state), device time from CUDA
events on the library's stream, max over ranks.  The plain FP64 step is timed
the same way on the same bar ("fp64"), and the per-field difference between
the two end states is reported ("accuracy").  e2e: the headline metric
through the split C-ABI entry points a Fortran driver calls (mcm_gpu_upload,
step_a/b/c per step with host dt logic, mcm_gpu_download), host buffers,
wall clock.  Each rank owns one independent bar (weak scaling, no data-path
collective).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
from mcmtop_b200 import ranks  # noqa: E402  (no CUDA work at import)
from mcmtop_b200.ranks import job_rate, max_over_ranks  # noqa: E402
# The batched ensemble runs bodies on up to 64 streams; give the CUDA context
# (created later, on first use) more hardware queues than the default 8.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

METRIC = "particle-steps/s (2M Taylor bar), mixed vs FP64 GPU at ≤1e-4 rel err; adj/fwd"
UNIT = "particle-steps/s"
DX = 0.08e-3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "exact", "mixed"])
    ap.add_argument("--no-compare", action="store_true", help="skip the FP64 run next to the mixed one")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint cost measurement")
    ap.add_argument("--adj-dx", type=float, default=0.2e-3, help="particle spacing of the differentiated bar")
    ap.add_argument("--adj-steps", type=int, default=400)
    ap.add_argument("--adj-every", type=int, default=50, help="checkpoint interval")
    ap.add_argument("--ens-bodies", type=int, default=256, help="bars of the batched ensemble (0: skip it)")
    ap.add_argument("--ens-steps", type=int, default=500)
    ap.add_argument("--ens-adj-steps", type=int, default=40,
                    help="steps of the ensemble's per-body gradients, batched and body after body (0: skip)")
    ap.add_argument("--ens-adj-every", type=int, default=10, help="checkpoint interval of the ensemble gradients")
    ap.add_argument("--fluid-steps", type=int, default=20, help="iterations of the 15.6M fluid column (0: skip)")
    ap.add_argument("--long-steps", type=int, default=2000,
                    help="iterations of the 2000-step accuracy run of the configuration, mixed, FP64-fast and "
                         "plain FP64 (0: skip)")
    ap.add_argument("--long-every", type=int, default=250, help="steps between the accuracy run's comparisons")
    ap.add_argument("--skin", type=float, default=0.0,
                    help="neighbour-list skin as a fraction of hmax for the FP64-fast and mixed runs (0: rebuild "
                         "the lists every step)")
    ap.add_argument("--pair-kind", type=int, default=0, choices=[0, 1, 2],
                    help="mixed gathers: 1 records through L1, 2 rows staged in shared memory (0: default)")
    ap.add_argument("--compensated", action="store_true",
                    help="mixed precision: Kahan-compensated pair sums per lane (compensated_sums)")
    ap.add_argument("--dx", type=float, default=DX)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=30.0, help="seconds of timed oracle work")
    ap.add_argument("--oracle-steps", type=int, default=20,
                    help="timed oracle steps on the full bar (the CPU baseline sample)")
    ap.add_argument("--oracle-check-steps", type=int, default=50,
                    help="oracle steps on the full bar for the GPU accuracy spot check")
    ap.add_argument("--reorder", type=int, default=20, help="steps between particle re-sorts")
    ap.add_argument("--long-only", type=int, default=-1, metavar="DEVICE",
                    help="run only the long accuracy run on this device and print its JSON (the child process "
                         "that the long-run leg starts)")
    ap.add_argument("--search-kind", type=int, default=0, choices=[0, 1, 2, 3],
                    help="neighbour search: 1 one thread per particle, 2 one warp per particle, 3 one warp per cell (0: default)")
    return ap.parse_args()


def device_clean(label: str) -> None:
    """Raises if a device error is pending at the point `label` (an
    asynchronous fault of an earlier leg would otherwise surface in the next
    leg's first synchronising call)."""
    import torch

    try:
        torch.cuda.synchronize()
    except Exception as exc:
        raise RuntimeError(f"device error pending at {label}: {exc}") from exc


def dist_env():
    return ranks.dist_env()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------- roofline
def algorithmic_bytes(region: str, kbar: float, precision: str, skin: bool = False) -> float:
    """Compulsory bytes per particle of one kernel group: the particle's own
    state read and written plus its neighbour list (4-byte entries), with
    ideal caching of the neighbour gathers (they count zero, as do sorts,
    gather records and other intermediates).  All state is FP64 in both
    precisions (the mixed path differs in its pair arithmetic).
      search:       read x(3) h mat; write count, list                 36 + 4 + 4K
      strain:       read x(3) v(3) m rho h, count, list                 72 + 4 + 4K
      constitutive: read v(3) m h rho e p c efps pcut fail sigma(6) rod(6) spin(3) tr vabs;
                    write x(3) rho e p c efps pcut sigma(6) q          224 + 8 + 136
      momentum:     read x v (6) m rho h sigma(6) q e vabs dispbc, count, list;
                    write x v (6) vabs                                 136 + 4 + 4 + 4K + 56
    With skin lists the search group also reads the positions of the last
    build (24) and at least K entries of the skin list (4K)."""
    if region == "search":
        return 36 + 4 + 4 * kbar + ((24 + 4 * kbar) if skin else 0.0)
    if region == "strain":
        return 72 + 4 + 4 * kbar
    if region == "constitutive":
        return 224 + 8 + 136
    if region == "momentum_integrate":
        return 136 + 4 + 4 + 4 * kbar + 56
    return 0.0


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(workload: str, precision: str, region: str):
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        d = json.load(fh)
    return d.get(workload, {}).get(precision, {}).get(region)


# -------------------------------------------------------------- CPU baseline
def cpu_oracle(deck, budget_s: float, max_steps: int, warmup: int = 0):
    """Times the OpenMP build of the CPU restatement (oracle/) on the deck:
    initialisation and `warmup` whole steps untimed (bounded by the budget),
    then whole steps until max_steps or the budget.  Returns the oracle as
    well, for the comparison with the GPU runs."""
    from oracle.pyoracle import Oracle

    orc = Oracle(deck, openmp=True)
    t0 = time.perf_counter()
    for _ in range(warmup):
        orc.run(1)
        if time.perf_counter() - t0 > budget_s:
            break
    steps = 0
    t0 = time.perf_counter()
    while steps < max_steps:
        orc.run(1)
        steps += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return deck.np * steps / el, steps, el, cores, orc


def advance_oracle(orc, done: int, target: int, budget_s: float) -> int:
    """Runs the oracle on from step `done` towards `target` steps (untimed,
    bounded by budget_s); returns the steps it has then run."""
    t0 = time.perf_counter()
    while done < target and time.perf_counter() - t0 < budget_s:
        orc.run(1)
        done += 1
    return done


ORACLE_FIELDS = ["x", "v", "rho", "e", "p", "c", "efps", "sigma", "q", "vabs"]


def oracle_spot_check(deck, orc, nsteps: int, local: int, reorder: int):
    """Per-field error of the mixed and the FP64 GPU steps against the FP64
    CPU oracle on the full bar after the oracle's first nsteps steps:
    max |gpu - oracle| / max |oracle| per field."""
    from mcmtop_b200 import _abi
    from mcmtop_b200.solver import Solver

    ref = {f: orc.get(f) for f in ORACLE_FIELDS}
    out = {"against": "FP64 CPU oracle (OpenMP build), same deck, first steps after initialisation",
           "steps": nsteps, "norm": "max |gpu - oracle| / max |oracle| per field"}
    for name, prec in (("mixed", _abi.PREC_MIXED), ("fp64", _abi.PREC_FP64)):
        s = Solver(deck, prec, device=local, reorder_interval=reorder)
        s.set_diagnostics(False)
        s.run(nsteps)
        g = s.download(ORACLE_FIELDS)
        s.close()
        err = {}
        for f in ORACLE_FIELDS:
            scale = float(np.max(np.abs(ref[f])))
            err[f] = float(np.max(np.abs(g[f] - ref[f])) / scale) if scale > 0 else float(np.max(np.abs(g[f])))
        out[name] = {"max_rel_err": {k: float(f"{v:.3e}") for k, v in err.items()},
                     "worst": float(f"{max(err.values()):.3e}")}
    return out


def adjoint_cost(args, local):
    """Gradient of a final-state function through the whole run against the
    forward run: the differentiated Taylor bar (FP64, prescribed dt schedule
    recorded from a nominal run, checkpoints every --adj-every steps).  All
    times are wall clock around synchronous ABI calls."""
    from mcmtop_b200 import _abi
    from mcmtop_b200.deck import taylor_bar
    from mcmtop_b200.solver import Solver

    deck = taylor_bar(dx=args.adj_dx)
    nsteps = args.adj_steps
    rec = Solver(deck, _abi.PREC_FP64, device=local)
    rec.set_diagnostics(False)
    dts = [rec.dt]
    for _ in range(nsteps):
        rec.step_a()
        rec.dt_update()
        dts.append(rec.dt)
        rec.step_b()
        rec.step_c()
    rec.close()
    fwd = Solver(deck, _abi.PREC_FP64, device=local)
    fwd.set_diagnostics(False)
    fwd.run(3)
    fwd.close()
    fwd = Solver(deck, _abi.PREC_FP64, device=local)
    fwd.set_diagnostics(False)
    t0 = time.perf_counter()
    done = fwd.run(nsteps)
    t_fwd = time.perf_counter() - t0
    fwd.close()
    # One untimed gradient on the same handle first: the first call allocates
    # the checkpoints and step records and loads the reverse kernels.  The
    # timed call then starts again from the uploaded initial state.
    sol = Solver(deck, _abi.PREC_FP64, device=local)
    init = sol.download()

    def gradient():
        sol.upload(init)
        t0 = time.perf_counter()
        sol.adjoint_forward(dts, args.adj_every)
        t_ckpt = time.perf_counter() - t0
        x = sol.download(["x"])["x"]
        xbar = np.zeros_like(x)
        z = x[:, 2]
        xbar[int(z.argmax()), 2] += 1.0   # d(final length)
        xbar[int(z.argmin()), 2] -= 1.0
        t0 = time.perf_counter()
        pb, _, _ = sol.adjoint_backward(xbar, None)
        return pb, t_ckpt, time.perf_counter() - t0

    pb_warm, _, _ = gradient()
    pb, t_ckpt, t_bwd = gradient()
    sol.close()
    spread = float(np.max(np.abs(pb - pb_warm) / np.maximum(np.abs(pb), 1e-300)))
    # the same gradient along the mixed-precision (FP32 pair sum) forward
    mixed = Solver(deck, _abi.PREC_MIXED, device=local)
    mixed.adjoint_forward(dts, args.adj_every)
    xm = mixed.download(["x"])["x"]
    xbar_m = np.zeros_like(xm)
    xbar_m[int(xm[:, 2].argmax()), 2] += 1.0
    xbar_m[int(xm[:, 2].argmin()), 2] -= 1.0
    pb32, _, _ = mixed.adjoint_backward(xbar_m, None)
    mixed.close()
    diff32 = float(np.max(np.abs(pb32 - pb) / np.maximum(np.abs(pb), 1e-300)))
    return {"workload": f"taylor_bar_{deck.np}", "steps": nsteps, "forward_steps_done": done,
            "checkpoint_every": args.adj_every, "precision": "fp64",
            "forward_s": round(t_fwd, 4), "forward_with_checkpoints_s": round(t_ckpt, 4),
            "backward_s": round(t_bwd, 4), "adj_over_fwd": round((t_ckpt + t_bwd) / t_fwd, 3),
            "backward_over_fwd": round(t_bwd / t_fwd, 3),
            "dlength_dparams": {"G": float(pb[0][0]), "yield": float(pb[0][1]), "hardening": float(pb[0][2]),
                                "eos_s": float(pb[0][3])},
            "repeat_rel_diff": spread,
            "fp32_forward": {"dlength_dparams": {"G": float(pb32[0][0]), "yield": float(pb32[0][1]),
                                                  "hardening": float(pb32[0][2]), "eos_s": float(pb32[0][3])},
                             "max_rel_diff_vs_fp64": diff32,
                             "note": "the same reverse kernels along the mixed-precision forward trajectory"},
            "note": "forward = fused mcm_gpu_run; gradient = checkpointed forward + reverse sweep, timed on the "
                    "second gradient of the handle (the first allocates its storage); parameter sums use atomics, "
                    "so repeated gradients differ in the last bits (repeat_rel_diff)"}


def fluid_column_cost(args, local):
    """The weakly compressible column collapse at full size: a 0.5 x 0.25 x 1.0 m
    block of water-like null material (linear polynomial EOS, c0 = 40 m/s) at
    dx = 2 mm (15.6 M particles) in a 2.0 x 0.25 x 1.2 m box of five ghost-
    particle walls, under gravity; headline precision, device time of
    --fluid-steps fused iterations after 3 warm-up iterations."""
    from mcmtop_b200 import _abi
    from mcmtop_b200.deck import fluid_column
    from mcmtop_b200.solver import Solver

    prec = {"fp64": _abi.PREC_FP64, "exact": _abi.PREC_FP64_EXACT, "mixed": _abi.PREC_MIXED}[args.precision]
    deck = fluid_column(dx=2.0e-3)
    s = Solver(deck, prec, device=local, reorder_interval=args.reorder)
    s.set_diagnostics(False)
    s.run(3)
    s.timer_start()
    done = s.run(args.fluid_steps)
    ms = s.timer_stop()
    st = s.stats()
    s.close()
    return {"workload": f"fluid_column_{deck.np}", "particles": deck.np, "steps": done, "precision": args.precision,
            "value": round(deck.np * done / (ms / 1e3), 1), "unit": UNIT, "ms_per_step": round(ms / max(done, 1), 3),
            "mean_neighbours": round(st["mean_nbr"], 2), "ghosts": st["ngp"],
            "note": "null material + EOS 1, five symmetry-plane walls of ghost particles, gravity; lists rebuilt "
                    "every step; device time (CUDA events on the library stream)"}


def ensemble_gradients(args, local, decks, prec, lanes, barrier=None):
    """Config 5's per-body gradients: for every body of this rank's block,
    d(final bar length)/d(G, yield stress, hardening modulus, EOS-41 s)
    through --ens-adj-steps steps of the headline precision (FP64 reverse
    kernels), checkpoints every --ens-adj-every steps, along each body's own
    dt schedule (recorded from a batched run of the same bodies).  Timed once
    as a batch (mcm_gpu_batch_adjoint_forward/backward) and once body after
    body (mcm_gpu_adjoint_forward/backward), from fresh handles both times
    (each includes the first allocation of its checkpoints); wall clock."""
    from mcmtop_b200.solver import Batch, Solver

    S, every = args.ens_adj_steps, args.ens_adj_every
    rec = [Solver(d, prec, device=local) for d in decks]
    for s in rec:
        s.set_diagnostics(False)
    rb = Batch(rec, lanes=lanes)
    dts = [[s.dt] for s in rec]
    for _ in range(S):
        rb.run(1)
        for k, s in enumerate(rec):
            dts[k].append(s.dt)
    rb.close()
    for s in rec:
        s.close()

    def length_adjoint(x):
        xbar = np.zeros_like(x)
        xbar[int(x[:, 2].argmax()), 2] += 1.0
        xbar[int(x[:, 2].argmin()), 2] -= 1.0
        return xbar

    bodies = [Solver(d, prec, device=local) for d in decks]
    if barrier:
        barrier()
    t0 = time.perf_counter()
    bb = Batch(bodies, lanes=lanes)
    bb.adjoint_forward(dts, every)
    xbars = [length_adjoint(s.download(["x"])["x"]) for s in bodies]
    pb, _, _ = bb.adjoint_backward(xbars, None)
    t_batch = time.perf_counter() - t0
    bb.close()
    for s in bodies:
        s.close()
    worst = 0.0
    t_seq = 0.0
    for k, d in enumerate(decks):
        s = Solver(d, prec, device=local)
        t0 = time.perf_counter()
        s.adjoint_forward(dts[k], every)
        pa, _, _ = s.adjoint_backward(length_adjoint(s.download(["x"])["x"]), None)
        t_seq += time.perf_counter() - t0
        s.close()
        worst = max(worst, float(np.max(np.abs(pb[k] - pa)) / max(float(np.max(np.abs(pa))), 1e-300)))
    return {"gradients": len(decks), "steps": S, "checkpoint_every": every, "loss": "final bar length",
            "params": ["G", "yield", "hardening", "eos_s"], "batched_s": t_batch, "sequential_s": t_seq,
            "max_rel_diff_batched_vs_alone": worst,
            "note": "forward in the headline precision, FP64 reverse kernels; batched = worker threads over the "
                    "bodies, each on its own stream; ghost-parent adjoints are summed with atomics, so batched "
                    "and alone agree to the last bits, not bitwise"}


def ensemble_cost(args, local, ws=1, rank=0, barrier=None):
    """The calibration ensemble: --ens-bodies independent Taylor bars (radius
    2-4 mm, L/D 6-12, 4k-64k particles log-uniform, yield 200-600 MPa, impact
    120-250 m/s) advanced --ens-steps iterations in the headline precision,
    once as a batch (one CUDA-graph launch per iteration of all bodies, lane
    count from mcm_gpu_batch_autotune) and once body after body through
    mcm_gpu_run, from the same initial states.  Wall clock around the
    synchronous calls; the end states of the two runs are compared.  With
    several ranks each rank advances its contiguous block of the bodies
    (ranks.share), the times are the slowest rank's, the work and the final
    bar lengths are gathered from every rank."""
    from mcmtop_b200 import _abi
    from mcmtop_b200.deck import taylor_ensemble
    from mcmtop_b200.ranks import gather_items, share, sum_over_ranks
    from mcmtop_b200.solver import Batch, Solver

    prec = {"fp64": _abi.PREC_FP64, "exact": _abi.PREC_FP64_EXACT, "mixed": _abi.PREC_MIXED}[args.precision]
    everyone = taylor_ensemble(nbodies=args.ens_bodies, seed=2024)
    mine = share(len(everyone), ws, rank)
    decks = [everyone[k] for k in mine]
    n_total = sum(d.np for d in everyone)
    dev = f"cuda:{local}"
    t0 = time.perf_counter()
    batched = [Solver(d, prec, device=local) for d in decks]
    t_init = time.perf_counter() - t0
    for s in batched:
        s.set_diagnostics(False)
    batch = Batch(batched, lanes=8)
    lanes, tuned_ms = batch.autotune(2)
    if barrier:
        barrier()
    t0 = time.perf_counter()
    done = batch.run(args.ens_steps)
    t_batch = max_over_ranks(time.perf_counter() - t0, dev)
    batch.close()
    seq = [Solver(d, prec, device=local) for d in decks]
    for s in seq:
        s.set_diagnostics(False)
    if barrier:
        barrier()
    t0 = time.perf_counter()
    done_seq = [s.run(args.ens_steps) for s in seq]
    t_seq = max_over_ranks(time.perf_counter() - t0, dev)
    same = all(np.array_equal(a.download(["x"])["x"], b.download(["x"])["x"]) for a, b in zip(batched, seq))
    lengths = {}
    for k, s in zip(mine, batched):
        z = s.download(["x"])["x"][:, 2]
        lengths[k] = float(z.max() - z.min())
    steps = int(sum_over_ranks(float(np.sum(done)), dev))
    work = sum_over_ranks(float(sum(d.np * int(k) for d, k in zip(decks, done))), dev)
    same_all = sum_over_ranks(0.0 if same else 1.0, dev) == 0.0
    final_len = gather_items(lengths, len(everyone), dev)[:, 0]
    for s in batched + seq:
        s.close()
    grads = ensemble_gradients(args, local, decks, prec, lanes, barrier) if args.ens_adj_steps > 0 else None
    if grads is not None:
        grads["batched_s"] = round(max_over_ranks(grads["batched_s"], dev), 3)
        grads["sequential_s"] = round(max_over_ranks(grads["sequential_s"], dev), 3)
        grads["speedup"] = round(grads["sequential_s"] / grads["batched_s"], 3)
        grads["gradients"] = int(sum_over_ranks(float(grads["gradients"]), dev))
        grads["max_rel_diff_batched_vs_alone"] = max_over_ranks(grads["max_rel_diff_batched_vs_alone"], dev)
    return {"workload": f"taylor_ensemble_{len(everyone)}x_{n_total}", "bodies": len(everyone),
            "particles": n_total, "ranks": ws, "bodies_per_rank": [len(share(len(everyone), ws, r)) for r in range(ws)],
            "particles_min": min(d.np for d in everyone), "particles_max": max(d.np for d in everyone),
            "steps": args.ens_steps, "body_steps_done": steps, "precision": args.precision,
            "lanes": lanes, "tuned_ms_per_step": round(tuned_ms, 4),
            "batched_s": round(t_batch, 3), "sequential_s": round(t_seq, 3),
            "batched_particle_steps_per_s": round(work / t_batch, 1),
            "sequential_particle_steps_per_s": round(work / t_seq, 1),
            "speedup": round(t_seq / t_batch, 3), "same_end_positions": bool(same_all),
            "sequential_done_equal": bool(list(done_seq) == [int(k) for k in done]),
            "final_length_cm": {"min": round(float(final_len.min()), 6), "max": round(float(final_len.max()), 6)},
            "init_s_per_body": round(t_init / max(len(decks), 1), 4),
            "gradients": grads,
            "note": "batched = mcm_gpu_batch_run (graph of one iteration of every body over the tuned lanes); "
                    "sequential = mcm_gpu_run per body, one after the other; wall clock, slowest rank; "
                    "each rank advances its contiguous block of the bodies"}


def long_run(args, local):
    """The configuration's full run: the bar advanced --long-steps iterations
    as the plain FP64 step (reference expressions and order), the FP64-fast
    step and the mixed step from the same initial state, in blocks of
    --long-every steps.  After each block, per field, the largest and the
    root-mean-square difference from the plain FP64 state (relative to the
    field's largest magnitude) of the mixed and the FP64-fast states; at the
    end the relative difference of the final bar lengths and each run's device
    time (CUDA events on the library's stream)."""
    from mcmtop_b200 import _abi
    from mcmtop_b200.deck import taylor_bar
    from mcmtop_b200.solver import Solver

    deck = taylor_bar(dx=args.dx)
    fields = ["x", "v", "rho", "e", "p", "c", "efps", "sigma", "q", "vabs"]
    runs = {"exact": _abi.PREC_FP64_EXACT, "fp64": _abi.PREC_FP64, "mixed": _abi.PREC_MIXED}
    sols = {}
    for name, prec in runs.items():
        sols[name] = Solver(deck, prec, device=local, reorder_interval=args.reorder,
                            nbr_skin=args.skin if prec != _abi.PREC_FP64_EXACT else 0.0, compensated=args.compensated)
        sols[name].set_diagnostics(False)
        device_clean(f"the end of the long run's {name} handle set-up")
    ms = {name: 0.0 for name in runs}
    growth = []
    done = 0
    err = {}
    every = max(1, min(args.long_every, args.long_steps))
    while done < args.long_steps:
        k = min(every, args.long_steps - done)
        for name, sol in sols.items():
            sol.timer_start()
            if sol.run(k) != k:
                raise RuntimeError(f"{name} long run stopped at step {done}")
            ms[name] += sol.timer_stop()
        done += k
        ends = {name: sol.download(fields) for name, sol in sols.items()}
        ref = ends["exact"]
        err = {}
        for name in ("mixed", "fp64"):
            e_max, e_rms = {}, {}
            for f in fields:
                scale = float(np.max(np.abs(ref[f]))) or 1.0
                d = np.abs(ends[name][f] - ref[f]).reshape(deck.np, -1).max(axis=1) / scale
                e_max[f] = float(f"{d.max():.3e}")
                e_rms[f] = float(f"{np.sqrt(np.mean(d * d)):.3e}")
            err[name] = {"max_rel_err": e_max, "rms_rel_err": e_rms, "worst": max(e_max.values()),
                         "worst_rms": max(e_rms.values())}
        growth.append({"step": done, "mixed_worst": err["mixed"]["worst"], "mixed_worst_rms": err["mixed"]["worst_rms"],
                       "fp64_worst": err["fp64"]["worst"]})
    length = {}
    for name in runs:
        z = ends[name]["x"][:, 2]
        length[name] = float(z.max() - z.min())
    l0 = float(deck.x[:, 2].max() - deck.x[:, 2].min())
    over = [g["step"] for g in growth if g["mixed_worst"] > 1e-4]
    out = {"workload": f"taylor_bar_{deck.np}", "steps": args.long_steps, "every": every,
           "against": "the plain FP64 GPU step (FP64-exact: reference expressions and summation order)",
           "norm": "per field, over particles: max (or root mean square) of |run - plain FP64| / max |plain FP64|",
           "mixed": err["mixed"], "fp64_fast": err["fp64"], "growth": growth,
           "mixed_within_1e-4": not over, "mixed_first_block_beyond_1e-4": over[0] if over else None,
           "final_length_rel_diff": {n: float(f"{abs(length[n] - length['exact']) / length['exact']:.3e}")
                                     for n in ("mixed", "fp64")},
           "within_0.1_percent": abs(length["mixed"] - length["exact"]) / length["exact"] <= 1e-3,
           "length_over_initial": {n: round(length[n] / l0, 6) for n in runs},
           "ms_per_step": {n: round(ms[n] / args.long_steps, 4) for n in runs},
           "particle_steps_per_s": {n: round(deck.np * args.long_steps / (ms[n] / 1e3), 1) for n in runs},
           "mixed_over_fp64_exact": round(ms["exact"] / ms["mixed"], 3),
           "mixed_over_fp64_fast": round(ms["fp64"] / ms["mixed"], 3),
           "note": "differences from the plain FP64 step grow exponentially at the same rate for every "
                   "perturbation: the FP64-fast step (fused multiply-add, other summation order) starts at "
                   "1e-16 and the mixed step at 1e-7 of the fields' ranges; the bar's length, a global "
                   "observable, stays within the bound"}
    for sol in sols.values():
        sol.close()
    return out


# ----------------------------------------------------------------- GPU arm
def gpu_arm(args):
    import torch

    from mcmtop_b200 import _abi
    from mcmtop_b200.deck import taylor_bar
    from mcmtop_b200.solver import Solver

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    prec = {"fp64": _abi.PREC_FP64, "exact": _abi.PREC_FP64_EXACT, "mixed": _abi.PREC_MIXED}[args.precision]
    deck = taylor_bar(dx=args.dx)
    workload = f"taylor_bar_{deck.np}"
    skin = args.skin if prec != _abi.PREC_FP64_EXACT else 0.0
    sol = Solver(deck, prec, device=local, reorder_interval=args.reorder, nbr_skin=skin,
                 compensated=args.compensated)
    sol.set_diagnostics(False)
    if args.search_kind or args.pair_kind:
        sol.set_tuning(search_kind=args.search_kind, pair_kind=args.pair_kind)
    sol.run(args.warmup)
    stats = sol.stats()
    kbar = stats["mean_nbr"]

    def barrier():
        if ws > 1:
            import torch.distributed as dist

            dist.barrier()

    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    gpu_index = int(vis.split(",")[local]) if vis else local
    clocks = ClockSampler(gpu_index)
    builds0 = sol.skin_builds() if skin > 0 else 0
    barrier()
    sol.profile(True)
    clocks.start()
    sol.timer_start()
    done = sol.run(args.steps)
    ms = sol.timer_stop()
    builds_timed = (sol.skin_builds() - builds0) if skin > 0 else None
    clk = clocks.stop()
    launches = sol.kernel_launches()
    report = sol.profile_report()
    sol.profile(False)
    if done != args.steps:
        raise RuntimeError(f"run stopped after {done} of {args.steps} steps")
    device_clean("the end of the timed run")
    ms_max = max_over_ranks(ms, f"cuda:{local}")
    value = job_rate(deck.np * args.steps, ws, ms_max)

    # roofline of the dominant kernel group
    peak, peak_kind = load_peaks()
    main = {k: v for k, v in report.items() if k in ("search", "strain", "constitutive", "momentum_integrate")}
    dom = max(main, key=lambda k: main[k][0])
    dom_ms, dom_n = main[dom]
    per_launch_s = dom_ms / 1e3 / max(dom_n, 1)
    bpp = algorithmic_bytes(dom, kbar, args.precision, skin > 0)
    achieved = bpp * deck.np / per_launch_s / 1e9
    traffic = load_traffic(workload, args.precision, dom)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "traffic": traffic, "bytes_per_particle": round(bpp, 1), "mean_neighbours": round(kbar, 2),
                "launch_ms": round(per_launch_s * 1e3, 4)}
    kernels = {k: {"ms_per_step": round(v[0] / args.steps, 4), "launches": v[1]} for k, v in report.items() if v[1]}

    # the plain FP64 step on the same bar, same steps; per-field difference of the end states
    fp64 = None
    accuracy = None
    if args.precision == "mixed" and not args.no_compare:
        ref = Solver(deck, _abi.PREC_FP64, device=local, reorder_interval=args.reorder, nbr_skin=skin)
        ref.set_diagnostics(False)
        if args.search_kind:
            ref.set_tuning(search_kind=args.search_kind)
        ref.run(args.warmup)
        barrier()
        ref.timer_start()
        done64 = ref.run(args.steps)
        ms64 = ref.timer_stop()
        ms64 = max_over_ranks(ms64, f"cuda:{local}")
        if done64 != args.steps:
            raise RuntimeError(f"FP64 run stopped after {done64} of {args.steps} steps")
        v64 = job_rate(deck.np * args.steps, ws, ms64)
        fp64 = {"value": round(v64, 1), "ms_per_step": round(ms64 / args.steps, 4),
                "mixed_over_fp64": round(value / v64, 3),
                "note": "FP64 with fused multiply-add and cooperative gathers (the optimised FP64 step)"}
        if rank == 0:
            fields = ["x", "v", "rho", "e", "p", "c", "efps", "sigma", "q", "vabs"]
            a_ = sol.download(fields)
            b_ = ref.download(fields)
            err = {}
            for f in fields:
                scale = float(np.max(np.abs(b_[f])))
                err[f] = float(np.max(np.abs(a_[f] - b_[f])) / scale) if scale > 0 else float(np.max(np.abs(a_[f])))
            la = a_["x"][:, 2].max() - a_["x"][:, 2].min()
            lb = b_["x"][:, 2].max() - b_["x"][:, 2].min()
            accuracy = {"against": "FP64 GPU step (itself within 1e-9 of the FP64 oracle in the parity tests)",
                        "steps": args.warmup + args.steps, "norm": "max |mixed - fp64| / max |fp64| per field",
                        "max_rel_err": {k: float(f"{v:.3e}") for k, v in err.items()},
                        "worst": float(f"{max(err.values()):.3e}"),
                        "length_rel_diff": float(f"{abs(la - lb) / lb:.3e}")}
        ref.close()
        device_clean("the end of the FP64-fast comparison")
        # the plain FP64 step: the reference's expressions and summation order,
        # no fused multiply-add, one thread per particle (MCM_PREC_FP64_EXACT)
        ex = Solver(deck, _abi.PREC_FP64_EXACT, device=local, reorder_interval=args.reorder)
        ex.set_diagnostics(False)
        if args.search_kind:
            ex.set_tuning(search_kind=args.search_kind)
        ex.run(args.warmup)
        barrier()
        ex.timer_start()
        done_ex = ex.run(args.steps)
        ms_ex = max_over_ranks(ex.timer_stop(), f"cuda:{local}")
        ex.close()
        device_clean("the end of the plain FP64 comparison")
        if done_ex != args.steps:
            raise RuntimeError(f"FP64-exact run stopped after {done_ex} of {args.steps} steps")
        v_ex = job_rate(deck.np * args.steps, ws, ms_ex)
        fp64["exact"] = {"value": round(v_ex, 1), "ms_per_step": round(ms_ex / args.steps, 4),
                         "mixed_over_fp64_exact": round(value / v_ex, 3),
                         "note": "the plain FP64 step: reference expressions and summation order, no fused "
                                 "multiply-add, one thread per particle"}

    ensemble = None
    if args.ens_bodies > 0:
        # every rank advances its block of the bodies; collectives in the same order on all ranks
        ensemble = ensemble_cost(args, local, ws, rank, barrier)

    # end to end through the split C ABI with host buffers (rank 0 only)
    e2e = None
    if rank == 0 and not args.no_e2e:
        names = ["x", "v", "mass", "h", "hold", "rho", "e", "p", "c", "vabs", "efps", "pcut", "fail", "sigma", "q",
                 "mat", "dispbc"]
        host = sol.download(names)
        # the host buffers a Fortran driver holds: pinned, in the ABI's layout
        # ((3,np) vectors, (3,3,np) column-major tensors), filled before the clock starts
        pinned = {}
        for k, a in host.items():
            src = np.ascontiguousarray(a.transpose(0, 2, 1) if a.ndim == 3 else a)
            t = torch.empty(src.shape, dtype=torch.from_numpy(src[:1].copy()).dtype, pin_memory=True)
            arr = t.numpy()
            arr[...] = src
            pinned[k] = arr
        bbox = np.array([host["x"][:, d].min() if j == 0 else host["x"][:, d].max() for d in range(3) for j in range(2)])
        h2d_bytes = sum(a.nbytes for a in pinned.values())
        k_e2e = args.steps
        # and the buffers the results come back into, also pinned
        out = {}
        for k in ["x", "v", "rho", "e", "p", "sigma", "efps"]:
            w = {"x": 3, "v": 3, "sigma": 9}.get(k, 1)
            out[k] = torch.empty((deck.np, w) if w > 1 else (deck.np,), dtype=torch.float64, pin_memory=True).numpy()
        t0 = time.perf_counter()
        sol.upload(pinned, bbox, fortran_layout=True)
        t1 = time.perf_counter()
        for k in range(k_e2e):
            # the energy sums are read at the output time (the last step), as a
            # driver writing time histories at output cadence does
            sol.step(energies=(k == k_e2e - 1))
        t2 = time.perf_counter()
        sol.download_into(out)
        el = time.perf_counter() - t0
        split_ms = {"upload": round((t1 - t0) * 1e3, 2), "steps": round((t2 - t1) * 1e3, 2),
                    "download": round((time.perf_counter() - t2) * 1e3, 2)}
        d2h_bytes = sum(a.nbytes for a in out.values())
        per_step_h2d = 24
        per_step_d2h = 96 + 8 * (5 * sol.nmat + 3) // k_e2e   # status + time at step_a; energies once
        e2e = {"value": round(deck.np * k_e2e / el, 1), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d_bytes / k_e2e + per_step_h2d),
               "d2h_bytes_per_step": int(d2h_bytes / k_e2e + per_step_d2h),
               "steps": k_e2e, "wall_ms": split_ms,
               "path": "mcm_gpu_upload + (step_a -> critts, host dt, step_b, step_c) x K + mcm_gpu_download; "
                       "step_a waits for the critical timestep while the step's momentum sum runs; step_b "
                       "returns the energies at the last step (the output time)"}

    adjoint = None
    if rank == 0 and not args.no_adjoint:
        device_clean("the start of the adjoint leg")
        adjoint = adjoint_cost(args, local)

    fluid = None
    if rank == 0 and args.fluid_steps > 0:
        device_clean("the start of the fluid-column leg")
        fluid = fluid_column_cost(args, local)

    longrun = None
    if rank == 0 and args.long_steps > 0 and args.precision == "mixed":
        device_clean("the start of the long run")
        longrun = long_run_in_child(args, local)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, n, el, cores, orc = cpu_oracle(deck, args.cpu_budget, args.oracle_steps)
        cpu = {"value": round(v, 1), "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"oracle (C++ restatement, OpenMP) on the same {deck.np}-particle bar: {n} steps after "
                         f"initialisation, {el:.1f} s"}
        if accuracy is not None:
            # the spot check runs the oracle on to --oracle-check-steps (the first 50)
            m = advance_oracle(orc, n, args.oracle_check_steps, 150.0)
            accuracy["vs_oracle"] = oracle_spot_check(deck, orc, m, local, args.reorder)
        orc.close()

    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": {"fp64": "f64", "exact": "f64", "mixed": "f32+f64"}[args.precision],
        "data": "synthetic: seeded jittered cubic lattice (Taylor bar, cm-g-us deck), no dataset",
        "config": {"workload": workload, "particles": deck.np, "dx_mm": args.dx * 1e3, "precision": args.precision,
                   "material": "copper model 10 + Mie-Grueneisen EOS 41, h = 1.3 dx, CFL 0.3 (tcrit_opt 1)",
                   "l2": "inputs larger than L2 (state ~1 GB/GPU)", "parallelism": "one independent bar per GPU",
                   "reorder_interval": args.reorder, "nbr_skin": skin, "compensated_sums": bool(args.compensated),
                "skin_builds_in_timed_steps": builds_timed},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk, "gpu_launches": launches,
        "fp64": fp64, "accuracy": accuracy, "long_run": longrun, "adjoint": adjoint, "ensemble": ensemble,
        "fluid_column": fluid,
        "kernels": kernels,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    sol.close()
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from mcmtop_b200.deck import taylor_bar

    deck = taylor_bar(dx=args.dx)
    # a bounded sample: W untimed steps, then the next steps of the same bar
    # until K steps or ~2 minutes
    v, n, el, cores, orc = cpu_oracle(deck, 120.0, max(1, args.steps), warmup=args.warmup)
    orc.close()
    line = {
        "metric": METRIC, "value": round(v, 1), "unit": UNIT, "n_gpus": ws, "steps": n, "warmup": args.warmup,
        "ms_per_step": round(el * 1e3 / n, 2), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "impl": "reference",
        "data": "synthetic: seeded jittered cubic lattice (Taylor bar, cm-g-us deck), no dataset",
        "config": {"workload": f"taylor_bar_{deck.np}", "particles": deck.np, "dx_mm": args.dx * 1e3,
                   "precision": "fp64", "parallelism": "host cores (OpenMP)"},
        "cpu_baseline": {"value": round(v, 1), "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"oracle (C++ restatement of the Fortran, the reference cannot be compiled: no "
                                   f"Fortran compiler) on the {deck.np}-particle bar, {args.warmup} untimed steps, "
                                   f"then {n} timed steps, {el:.1f} s"},
        "e2e": {"value": round(v, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def long_run_in_child(args, local):
    """long_run in a process of its own, on the same GPU.  In one process,
    after the earlier legs had created and destroyed some hundreds of handles,
    the set-up of the long run's handles met an illegal memory access whose
    cause is not found; a fresh process (a fresh CUDA context) keeps that
    history away from the long run, and a failure of the child is recorded in
    the line instead of ending the whole measurement."""
    cmd = [sys.executable, os.path.abspath(__file__), "--long-only", str(local), "--dx", repr(args.dx),
           "--long-steps", str(args.long_steps), "--long-every", str(args.long_every), "--reorder", str(args.reorder),
           "--skin", repr(args.skin)] + (["--compensated"] if args.compensated else [])
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=1800)
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        tail = " | ".join(r.stderr.strip().splitlines()[-3:])
        return {"error": f"long run child exited {r.returncode}: {tail}"}
    out = json.loads(lines[-1])
    out["process"] = "child (own CUDA context)"
    return out


def main():
    args = parse()
    if args.long_only >= 0:
        print(json.dumps(long_run(args, args.long_only)))
        return
    if args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
