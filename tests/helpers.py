"""Shared test helpers: fixture loading and comparisons."""
import glob
import os

import numpy as np

from golden.make_golden import load_case  # noqa: F401  (re-exported)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
STAGED = ["cav4", "cav6j", "chan_sym", "cht", "cav4_opts", "cav4_global", "chan_massflow"]


def fixture_path(name: str) -> str:
    return os.path.join(GOLDEN, name + ".npz")


def all_fixtures():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def bitwise(a, b) -> bool:
    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype.kind == "f":
        return np.array_equal(a.view(np.int64), b.astype(np.float64).view(np.int64))
    return np.array_equal(a, b)


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def stage_step(z) -> int:
    """1-based step whose intermediate arrays the fixture holds (0 if none)."""
    return int(z["stage_step"][0])


def params_of(case) -> dict:
    return case.params
