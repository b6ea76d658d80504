"""Regenerates the Lobato & Van Dyck (2014) parameter table used by the CUDA library and the oracle.

The numbers are the (a_i, b_i), i = 1..5, per element Z = 1..103 that SimulatoKit ships in
`Sources/SimulatoMultislice/LobatoTable.swift:10-116` (abTEM 1.0.10's `lobato.json`, verbatim doubles). They are
physical data, kept identical on purpose so that f(k^2) agrees with the reference bit for bit.

Writes, from the one source:
  simulatokit_b200/data/lobato.json        (for the Python host code and the CPU oracle)
  simulatokit_b200/csrc/lobato_table.inc   (compiled into libsimulato_cuda.so)

Usage: python simulatokit_b200/data/make_lobato_table.py path/to/Sources/SimulatoMultislice/LobatoTable.swift
(the file of a SimulatoKit checkout; required).
"""

from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def parse(text: str) -> list[tuple[int, str, list[float], list[float]]]:
    rows = []
    pat = re.compile(r"\(a: \[([^\]]*)\], b: \[([^\]]*)\]\), // (\d+) (\w+)")
    for m in pat.finditer(text):
        a = [float(x) for x in m.group(1).split(",")]
        b = [float(x) for x in m.group(2).split(",")]
        rows.append((int(m.group(3)), m.group(4), a, b))
    return rows


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: python simulatokit_b200/data/make_lobato_table.py path/to/LobatoTable.swift")
    src = sys.argv[1]
    rows = parse(open(src).read())
    assert [r[0] for r in rows] == list(range(1, 104)), "expected Z = 1..103 in order"
    assert all(len(r[2]) == 5 and len(r[3]) == 5 for r in rows)
    table = {"source": "Lobato & Van Dyck, Acta Cryst. A 70, 636-649 (2014), as shipped by abTEM 1.0.10",
             "elements": [{"Z": z, "symbol": s, "a": a, "b": b} for z, s, a, b in rows]}
    with open(os.path.join(HERE, "lobato.json"), "w") as fh:
        json.dump(table, fh, indent=0)
    lines = ["// Generated by simulatokit_b200/data/make_lobato_table.py; do not edit.",
             "// Lobato & Van Dyck (2014) parameters: {a1..a5, b1..b5} for Z = 1..103 (index Z - 1).",
             "static const double kLobatoTable[103][10] = {"]
    for z, s, a, b in rows:
        vals = ", ".join(repr(x) for x in a + b)
        lines.append(f"    {{{vals}}},  // {z} {s}")
    lines.append("};")
    with open(os.path.join(HERE, "..", "csrc", "lobato_table.inc"), "w") as fh:
        fh.write("\n".join(lines) + "\n")
    print(f"wrote {len(rows)} elements")


if __name__ == "__main__":
    main()
