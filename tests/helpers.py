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


def read_vtu(path):
    """Arrays of a binary-appended (raw, UInt64 headers) VTU file by name;
    the points under 'Points'."""
    import re
    raw = open(path, "rb").read()
    head, _, rest = raw.partition(b"<AppendedData encoding=\"raw\">")
    data = rest[rest.index(b"_") + 1:]
    types = {"Float64": np.float64, "Int32": np.int32, "UInt8": np.uint8}
    out = {}
    for m in re.finditer(rb'<DataArray type="(\w+)"(?: Name="(\w+)")? NumberOfComponents="(\d+)" format="appended" offset="(\d+)"/>', head):
        t, name, nc, off = m.group(1).decode(), m.group(2), int(m.group(3)), int(m.group(4))
        n = int(np.frombuffer(data[off:off + 8], dtype=np.uint64)[0])
        a = np.frombuffer(data[off + 8:off + 8 + n], dtype=types[t])
        out[name.decode() if name else "Points"] = a.reshape(-1, nc) if nc > 1 else a
    cells = re.search(rb'NumberOfPoints="(\d+)" NumberOfCells="(\d+)"', head)
    out["_npoints"], out["_ncells"] = int(cells.group(1)), int(cells.group(2))
    return out
