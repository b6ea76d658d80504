"""Copies subsets of SimulatoKit's abTEM-generated float64 fixtures into tests/golden/.

Source: `Tests/SimulatoKitParityTests/Fixtures/*-pins.json` + `*-arrays.bin` of the SimulatoKit checkout (float64
little-endian, complex interleaved; sha256 recorded in each JSON and checked here, as the reference's loaders do,
`Tests/SimulatoKitParityTests/Multislice/Pins.swift:21-45`). The arrays kept are the ones the parity tests read;
the JSON scalars are kept whole (minus the array index). The GPU box has no reference checkout, so the tests read
only what this script writes.

Usage: python tests/golden/make_golden.py /path/to/SimulatoKit   (the checkout's root; required)
"""

from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

KEEP = {
    "slice-1": ["A1.V.0", "A1.t.0", "A1/plane.exit.0", "A1/plane.pattern.0",
                "A2.V.0", "A2/plane.exit.0",
                "D1.V.0", "D1.V.1", "D1.t.0", "D1/plane.exit.0", "D1/plane.pattern.0",
                "D1/probe.incident", "D1/probe.exit.0", "D1/probe.pattern.0",
                "B2/probe.incident"],
    "slice-2": None,   # all (1.4 MB)
    "slice-4": None,
    "slice-3": None,   # CTF kernels and HRTEM images (1.5 MB)
    "slice-4-scan": ["com_mrad", "com_inv", "dp", "dp_gauss", "dp_gauss_big"],
    "icom": None,      # gradient integrations, the scan's centre of mass and iCOM, disc and tile images (26 KB)
    "waves": None,     # all six runs (1.5 MB): full size and five Fourier resamplings
}


def load(root: str, name: str):
    fx = os.path.join(root, "Tests", "SimulatoKitParityTests", "Fixtures")
    pins = json.load(open(os.path.join(fx, f"{name}-pins.json")))
    blob = open(os.path.join(fx, pins["arrays"]["file"]), "rb").read()
    assert hashlib.sha256(blob).hexdigest() == pins["arrays"]["sha256"], f"{name}: sha256 mismatch"
    arrays = {}
    for key, e in pins["arrays"]["index"].items():
        raw = np.frombuffer(blob, dtype="<f8", count=e["count"] * (2 if e["kind"] == "c16" else 1), offset=e["offset"])
        a = raw[0::2] + 1j * raw[1::2] if e["kind"] == "c16" else raw.copy()
        arrays[key] = a.reshape(e["shape"])
    meta = {k: v for k, v in pins.items() if k != "arrays"}
    meta["source_sha256"] = pins["arrays"]["sha256"]
    return meta, arrays


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/SimulatoKit")
    root = sys.argv[1]
    all_meta = {}
    for name, keep in KEEP.items():
        meta, arrays = load(root, name)
        meta.pop("self_checks", None)
        all_meta[name] = meta
        sel = arrays if keep is None else {k: arrays[k] for k in keep}
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **{k.replace("/", "__"): v for k, v in sel.items()})
        print(name, len(sel), "arrays")
    with open(os.path.join(HERE, "pins.json"), "w") as fh:
        json.dump(all_meta, fh, indent=0, sort_keys=True)


if __name__ == "__main__":
    main()
