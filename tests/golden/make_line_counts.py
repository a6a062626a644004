"""Writes reference_line_counts.json: the number of lines of every Fortran
source of the reference (MarkoTopalovic/MCMtop, directory MCM/), so that the
citation test can check `file.f90:N` references without the reference tree.

    python tests/golden/make_line_counts.py /path/to/MCMtop
"""
import json
import os
import sys


def main(root: str) -> None:
    src = os.path.join(root, "MCM")
    counts = {}
    for name in sorted(os.listdir(src)):
        if name.lower().endswith(".f90"):
            with open(os.path.join(src, name), "rb") as fh:
                data = fh.read()
            counts[name] = data.count(b"\n") + (1 if data and not data.endswith(b"\n") else 0)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_line_counts.json")
    with open(out, "w") as fh:
        json.dump(counts, fh, indent=0, sort_keys=True)
        fh.write("\n")
    print(f"{len(counts)} files -> {out}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
