"""Every `file.f90:N` citation in the repository's code and documents points
at lines that exist in the cited reference file.  The line counts come from
tests/golden/reference_line_counts.json (tests/golden/make_line_counts.py
writes it from a checkout of the reference)."""
import json
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
COUNTS = os.path.join(ROOT, "tests", "golden", "reference_line_counts.json")
# documents written by others (the survey, reviews, published baselines) are not checked
SKIP = {"SURVEY.md", "VERDICT.md", "ADVICE.md", "BASELINE.md", "BASELINE.json"}
EXT = (".py", ".cu", ".cuh", ".h", ".cpp", ".md", ".f90")
CITE = re.compile(r"\b([A-Za-z0-9_]+\.[fF]90):(\d+(?:-\d+)?(?:,\s?\d+(?:-\d+)?)*)")


def repo_files():
    for d, dirs, files in os.walk(ROOT):
        rel = os.path.relpath(d, ROOT)
        parts = rel.split(os.sep)
        if parts[0] in (".git", "_work", "gpurun_out", "baseline", "_build") or any(
                p.startswith(".") or p in ("__pycache__", "_build") for p in parts if p != "."):
            dirs[:] = []
            continue
        for f in files:
            if f.endswith(EXT) and not (rel == "." and f in SKIP):
                yield os.path.join(d, f)


def citations():
    for path in repo_files():
        with open(path, encoding="utf-8", errors="replace") as fh:
            for ln, line in enumerate(fh, 1):
                for m in CITE.finditer(line):
                    yield os.path.relpath(path, ROOT), ln, m.group(1), m.group(2)


def out_of_range():
    with open(COUNTS) as fh:
        counts = json.load(fh)
    lower = {k.lower(): v for k, v in counts.items()}
    bad, total = [], 0
    for path, ln, name, spans in citations():
        total += 1
        n = lower.get(name.lower())
        if n is None:
            bad.append((path, ln, f"{name}: no such reference file"))
            continue
        for span in spans.replace(" ", "").split(","):
            a, _, b = span.partition("-")
            lo, hi = int(a), int(b or a)
            if not (1 <= lo <= hi <= n):
                bad.append((path, ln, f"{name}:{span} (file has {n} lines)"))
    return bad, total


def test_reference_citations_exist():
    bad, total = out_of_range()
    assert total > 100
    assert not bad, "\n".join(f"{p}:{ln}: {msg}" for p, ln, msg in bad)
