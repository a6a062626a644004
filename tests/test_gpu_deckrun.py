"""A deck file run through the program loop (deck reader, GPU step, output
writers), against the same loop driven by the oracle."""
import os
import subprocess
import sys

import numpy as np
import pytest

from mcmtop_b200 import _abi
from mcmtop_b200.deck import taylor_bar
from mcmtop_b200.deckio import read_deck, write_deck
from mcmtop_b200.output import read_vtk
from mcmtop_b200.run import Program
from test_deckio import oracle_program

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STEPS = 40


def bar_deck(tmp_path, **kw):
    kw.setdefault("state_opt", 4)
    d = taylor_bar(dx=0.4e-3).replace(stpltime=0.5, thpltime=0.2, thnodes=(1, 8000, 16848),
                                      transducers=(((0.0, 0.0, 0.3), 1),), status_interval=25, title="taylor bar",
                                      **kw)
    path = tmp_path / "bar.mcm"
    write_deck(d, path)
    return read_deck(str(path)), path


def run_program(deck, directory, fuse, precision=_abi.PREC_FP64_EXACT, steps=STEPS):
    os.makedirs(directory, exist_ok=True)
    p = Program(deck, "bar", str(directory), precision, fuse=fuse)
    try:
        p.initial()
        n = p.run(steps)
        state = p.solver.download(["x", "v", "sigma", "rho", "e", "p"])
        return n, state, p.fused_steps, p.out
    finally:
        p.close()


def _files(directory):
    return {n: (directory / n).read_text() for n in sorted(os.listdir(directory))}


def test_fused_stretches_write_the_same_files(tmp_path, gpu_lib):
    deck, _ = bar_deck(tmp_path)
    na, sa, fused, out = run_program(deck, tmp_path / "fused", True)
    nb, sb, none, _ = run_program(deck, tmp_path / "stepwise", False)
    assert na == nb == STEPS and fused > 0 and none == 0
    for f in sa:
        assert np.array_equal(sa[f], sb[f]), f
    fa, fb = _files(tmp_path / "fused"), _files(tmp_path / "stepwise")
    assert fa.keys() == fb.keys() and out.istate >= 2
    for n in fa:
        assert fa[n] == fb[n], n


def _numbers(text, width12=False):
    out = []
    if width12:   # EnSight records: e12.5 fields that touch when negative
        for ln in text.splitlines():
            for k in range(0, len(ln), 12):
                try:
                    out.append(float(ln[k:k + 12]))
                except ValueError:
                    pass
        return np.array(out)
    for ln in text.splitlines():
        for tok in ln.replace(",", " ").split():
            try:
                out.append(float(tok))
            except ValueError:
                pass
    return np.array(out)


@pytest.mark.parametrize("state_opt", [4, 1], ids=["vtk", "ensight"])
def test_outputs_match_the_oracle_program(state_opt, tmp_path, gpu_lib, oracle_lib):
    deck, _ = bar_deck(tmp_path, state_opt=state_opt)
    run_program(deck, tmp_path / "gpu", True)
    os.makedirs(tmp_path / "cpu")
    orc, _ = oracle_program(deck, "bar", str(tmp_path / "cpu"), STEPS)
    orc.close()
    fg, fc = _files(tmp_path / "gpu"), _files(tmp_path / "cpu")
    assert fg.keys() == fc.keys()
    same = total = 0
    for n in fg:
        lg, lc = fg[n].splitlines(), fc[n].splitlines()
        assert len(lg) == len(lc), n
        same += sum(a == b for a, b in zip(lg, lc))
        total += len(lg)
        a, b = _numbers(fg[n], width12=not n.endswith((".csv", ".vtk"))), _numbers(fc[n], width12=not n.endswith((".csv", ".vtk")))
        assert a.shape == b.shape, n
        # printed with 5-8 significant digits: a last-digit flip at most
        scale = np.maximum(np.abs(b), 1e-300)
        assert np.all((np.abs(a - b) <= 2e-5 * scale) | (np.abs(a - b) <= 2e-8)), n
    assert same >= 0.999 * total, f"{total - same} of {total} output lines differ"


def test_vtk_holds_the_downloaded_state(tmp_path, gpu_lib):
    deck, _ = bar_deck(tmp_path, endtime=0.25)
    n, state, _, out = run_program(deck, tmp_path / "end", True, steps=None)
    # the run ends at the termination test, before the last velocity update,
    # and writes a state there (ptime >= endtime)
    last = out.istate - 1
    vt = read_vtk(str(tmp_path / "end" / f"bar{last}.vtk"))
    np.testing.assert_allclose(vt["x"], state["x"], rtol=0, atol=5.1e-9)
    np.testing.assert_allclose(vt["Stress_X"], state["sigma"][:, 0, 0], rtol=5e-5, atol=1e-300)


def test_mixed_precision_program(tmp_path, gpu_lib):
    deck, _ = bar_deck(tmp_path)
    n, state, fused, out = run_program(deck, tmp_path / "mixed", True, _abi.PREC_MIXED)
    assert n == STEPS and fused > 0 and np.isfinite(state["sigma"]).all()
    assert os.path.exists(tmp_path / "mixed" / "bar_th8000.csv")


def test_command_line(tmp_path, gpu_lib):
    _, path = bar_deck(tmp_path)
    r = subprocess.run([sys.executable, "-m", "mcmtop_b200", f"i={path}", "o=cli", f"dir={tmp_path}", "steps=30"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "Problem status for time-step     25" in r.stdout
    assert "State plot written at time" in r.stdout
    assert os.path.exists(tmp_path / "cli0.vtk") and os.path.exists(tmp_path / "cli_th16848.csv")
    log = (tmp_path / "cli.log").read_text()
    assert log.startswith("taylor bar") and "Problem status for time-step     25" in log
