"""Readers for the golden fixtures in tests/golden/ (subsets of SimulatoKit's abTEM float64 pins)."""

import functools
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@functools.lru_cache(maxsize=None)
def pins():
    return json.load(open(os.path.join(GOLDEN, "pins.json")))


@functools.lru_cache(maxsize=None)
def _npz(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def array(name, key):
    return _npz(name)[key.replace("/", "__")]


def case(name, key):
    return pins()[name]["cases"][key]
