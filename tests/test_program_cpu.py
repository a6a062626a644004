"""The program loop's host logic (no GPU): how many iterations may run fused
on the device before an output time, a status report or the end."""
import types

import numpy as np

from mcmtop_b200.run import Program, parse_args


class _Out:
    def __init__(self, t):
        self.t = t

    def next_time(self):
        return self.t


def _program(dt, ptime, next_time, timestep, status_interval, fuse=True):
    p = Program.__new__(Program)
    p.solver = types.SimpleNamespace(dt=dt, ptime=ptime, timestep=timestep)
    p.out = _Out(next_time)
    p.fuse = fuse
    p.status_interval = status_interval
    return p


def test_fused_stretch_never_reaches_an_output_time():
    rng = np.random.default_rng(11)
    for _ in range(2000):
        dt = 10.0 ** rng.uniform(-3, 0)
        ptime = rng.uniform(0, 10)
        gap = dt * 10.0 ** rng.uniform(-1, 3)
        ts = int(rng.integers(1, 10000))
        si = int(rng.integers(1, 200))
        p = _program(dt, ptime, ptime + gap, ts, si)
        k = p._safe_steps()
        # worst case: dt grows by 1.1 every iteration (MCM/mcm_solution.f90:61)
        t, d = ptime, dt
        for _ in range(k):
            d *= 1.1
            t += d
            assert t < ptime + gap
        for step in range(ts, ts + k):
            assert step % si != 0


def test_no_fusing_when_output_is_due_or_disabled():
    assert _program(1.0, 5.0, 5.0, 3, 100)._safe_steps() == 0
    assert _program(1.0, 5.0, 100.0, 3, 100, fuse=False)._safe_steps() == 0
    assert _program(1.0, 5.0, 100.0, 100, 100)._safe_steps() == 0   # a status step comes next


def test_command_line_arguments():
    a = parse_args(["i=bar", "o=out", "precision=mixed", "steps=5"])
    assert a == {"i": "bar", "o": "out", "precision": "mixed", "steps": "5"}
    for bad in (["o=out"], ["i=a", "i=b"], ["x"], ["i=a", "r=restart"]):
        try:
            parse_args(bad)
        except SystemExit:
            continue
        raise AssertionError(bad)
