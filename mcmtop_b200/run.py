"""The MCM program around the GPU step: read a deck, initialise, loop with
output, as MCM/main.f90 does (mcm_getinput, mcm_initial, mcm_solution).

    python -m mcmtop_b200 i=<deck> [o=<output name>] [precision=fp64|fast|mixed] [dir=<directory>]

reads ``<deck>.mcm`` (MCM/mcm_parse_cl.f90: arguments ``i=`` and ``o=``; the
output name defaults to the input name), runs to the deck's termination time
and writes the state, time-history and transducer files of the deck's
output options (mcmtop_b200.output).  The loop is MCM/mcm_solution.f90:37-138
through the split step (mcm_gpu_step_a/b/c); stretches of iterations in
which no output, status report or termination can occur run fused on the
device (mcm_gpu_run) with the same dt arithmetic.
"""
from __future__ import annotations

import os
import sys

from . import _abi
from .deckio import read_deck
from .output import Outputs, state_line, status_line
from .solver import Solver

PRECISIONS = {"fp64": _abi.PREC_FP64_EXACT, "exact": _abi.PREC_FP64_EXACT, "fast": _abi.PREC_FP64,
              "mixed": _abi.PREC_MIXED}


class Program:
    """One problem: Solver + Outputs + the loop of mcm_solution."""

    def __init__(self, deck, fileout: str, directory: str = ".", precision: int = _abi.PREC_FP64_EXACT,
                 echo=None, fuse: bool = True):
        self.deck = deck
        self.solver = Solver(deck, precision)
        self.out = Outputs(deck, fileout, directory)
        self.echo = echo
        self.fuse = fuse
        # MCM/mcm_control_v2.f90:198
        self.status_interval = deck.status_interval if deck.status_interval >= 1 else 100
        self.fused_steps = 0
        self.sync_steps = 0
        self.log = None

    def _say(self, text: str) -> None:
        """A message for the screen and the log file (MCM writes both, units * and 13)."""
        if self.echo:
            self.echo(text)
        if self.log is not None:
            self.log.write(text + "\n")

    def _state(self, fields) -> dict:
        return self.solver.download(list(fields)) if fields else {}

    def initial(self) -> None:
        """MCM/mcm_initial.f90:109-115: first state and time-history output."""
        fields = self.out.fields(True, True)
        self.out.initial(self.solver.ptime, self._state(fields), self.solver.energies_now())

    def _safe_steps(self) -> int:
        """Iterations that can run fused: every one of them must end with
        ptime below the next output time (dt grows at most by 1.1 per step,
        MCM/mcm_solution.f90:61) and none may be a status step."""
        s = self.solver
        gap = self.out.next_time() - s.ptime
        if not self.fuse or s.dt <= 0.0 or gap <= 0.0:
            return 0
        limit = gap * (1.0 - 1e-9)
        k, grow, total = 0, 1.0, 0.0
        while k < 100000:
            grow *= 1.1
            total += s.dt * grow
            if total >= limit:
                break
            k += 1
        to_status = (-s.timestep) % self.status_interval
        return min(k, to_status)

    def step(self, budget: int | None = None) -> bool:
        """Fused iterations that need no host (at most budget - 1 of them),
        then one loop iteration with its output; False once the run ends."""
        s = self.solver
        k = self._safe_steps()
        if budget is not None:
            k = min(k, budget - 1)
        if k > 0:
            done = s.run(k)
            self.fused_steps += done
            if done < k:
                raise RuntimeError("fused iterations ended early")
        s.step_a()
        s.dt_update()
        s.step_b()
        self.sync_steps += 1
        st, th = self.out.due(s.ptime)
        fields = self.out.fields(st, th)
        if st or th:
            cf = s.contact_forces() if (th and self.deck.contacttype > 0) else None
            self.out.after_energies(s.ptime, self._state(fields), s.energies, cf)
        if st:
            self._say(state_line(s.ptime))
        if s.timestep % self.status_interval == 0:
            self._say(status_line(s.timestep, s.ptime, s.dt))
        if s.ptime - s.dt >= self.deck.endtime:       # MCM/mcm_solution.f90:101
            s.ended = True
            return False
        s.step_c()
        return True

    def run(self, max_steps: int | None = None) -> int:
        """Runs to termination (or max_steps more iterations); returns the
        iterations done."""
        start = self.solver.timestep
        while max_steps is None or self.solver.timestep - start < max_steps:
            budget = None if max_steps is None else max_steps - (self.solver.timestep - start)
            if not self.step(budget):
                break
        return self.solver.timestep - start

    def finish(self) -> None:
        """MCM/main.f90: mcm_write_drelax after the loop has terminated."""
        if self.solver.ended:
            from .output import DRELAX_FIELDS
            self.out.drelax(self._state(DRELAX_FIELDS))

    def open_log(self) -> None:
        """<out>.log with the status and state-output messages (the reference's
        log also echoes the input cards, which this one does not)."""
        self.log = open(self.out.base + ".log", "w")
        self.log.write(f"{(self.deck.title or self.deck.name)[:78]}\n")

    def close(self) -> None:
        if self.log is not None:
            self.log.close()
            self.log = None
        self.solver.close()


def parse_args(argv) -> dict:
    """MCM/mcm_parse_cl.f90: each argument is <letter>=<value>; i= is required."""
    out = {}
    for a in argv:
        if len(a) < 2 or a[1] != "=" and not a.startswith(("precision=", "dir=", "steps=")):
            raise SystemExit(f"argument {a!r} is not of the form i=<input>, o=<output>, precision=, dir=, steps=")
        key, _, val = a.partition("=")
        if key in out:
            raise SystemExit(f"argument {key}= given twice")
        out[key] = val
    if "i" not in out:
        raise SystemExit("no input file given (i=<name>)")
    if "r" in out:
        raise SystemExit("restart files are not supported")
    return out


def main(argv=None) -> int:
    args = parse_args(sys.argv[1:] if argv is None else argv)
    name = args["i"]
    path = name if name.endswith(".mcm") else name + ".mcm"
    deck = read_deck(path)
    fileout = args.get("o", os.path.splitext(os.path.basename(name))[0])
    directory = args.get("dir", ".")
    prec = PRECISIONS[args.get("precision", "fp64")]
    prog = Program(deck, fileout, directory, prec, echo=print)
    try:
        prog.open_log()
        prog.initial()
        n = prog.run(int(args["steps"]) if "steps" in args else None)
        prog.finish()
        print(f"\n     {n} time steps, time {prog.solver.ptime:.6e}; "
              f"{prog.fused_steps} fused on the device, {prog.sync_steps} with host output checks")
    finally:
        prog.close()
    return 0
