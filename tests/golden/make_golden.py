"""Generates the golden fixtures of tests/golden/ by running the reference
solver itself (compiled from its own sources by oracle/Makefile into
oracle/_ref/cbs_ref_harness) on seeded synthetic cases with one OpenMP
thread, so every sum is in the reference's serial order.

Run here, where the reference sources exist:
    make -C oracle ref && python tests/golden/make_golden.py
Each fixture is an .npz holding the case description (mesh arrays and .par
parameters), the preprocessing arrays, every intermediate array of one
stage-dumped step, the per-step history and the final fields.
"""

from __future__ import annotations

import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "cbs-3d_b200"))
sys.path.insert(0, ROOT)

from cbs3d import cases  # noqa: E402
from oracle import pyoracle  # noqa: E402


def golden_cases():
    """name -> (case, nsteps, stage_step, every)"""
    return {
        "cav4": (cases.cavity(4, re=100.0, ntime=3), 3, 2, 0),
        "cav6j": (cases.cavity(6, re=400.0, ntime=5, jitter=0.15, seed=7), 5, 3, 0),
        "chan_sym": (cases.channel(8, 4, 4, length=2.0, re=100.0, ntime=4, symmetry_z=True), 4, 2, 0),
        "cht": (cases.cht_slab(8, 4, 2, 4, ntime=3, q=1.0), 3, 2, 0),
        "cav4_opts": (cases.cavity(4, re=250.0, ntime=4, htype=2, ilots=2, step2_check=1, deltr=0.05,
                                   cg_conv_test=3, absToler=1e-9), 4, 3, 0),
        "cav4_global": (cases.cavity(4, re=100.0, ntime=3, ilots=0, htype=3), 3, 2, 0),
        "chan_massflow": (_massflow_channel(), 3, 2, 0),
        "c1_cavity16": (cases.cavity(16, re=100.0, ntime=500), 500, 0, 100),
    }


def _massflow_channel():
    c = cases.channel(6, 3, 3, length=2.0, re=50.0, ntime=3)
    c.bc_map = {1: 511, 2: 520, 3: 530, 4: 501, 5: 502, 6: 530}
    c.params.update(temp_calc=1, massflow_enabled=1, mdot=0.5, rho_in=1.0, T_in=0.25)
    return c


# preprocessing arrays kept only in the small stage fixtures
_BULKY = {"dNkdx", "annxf", "gstifE", "pdiagE", "elcoe_e", "face_norm", "iside", "fedge", "detJ", "alen_e",
          "Mdiag_real", "mat_elem"}


def fixture_payload(case, ref: dict, nsteps: int, stage: int) -> dict:
    m = case.mesh
    out = {
        "intma": m.intma.astype(np.int32), "coord": m.coord, "bfaces": m.bfaces.astype(np.int32),
        "mat_elem": m.mat_elem.astype(np.int32),
        "bc_map": np.array(sorted(case.bc_map.items()), dtype=np.int32),
        "params_json": np.frombuffer(json.dumps(case.params, sort_keys=True).encode(), dtype=np.uint8),
        "materials_json": np.frombuffer(json.dumps({str(k): v for k, v in case.materials.items()}).encode(),
                                        dtype=np.uint8),
    }
    out["nsteps"] = np.array([nsteps], dtype=np.int32)
    out["stage_step"] = np.array([stage], dtype=np.int32)
    for k, v in ref.items():
        if k in ("coord", "intma") or (stage == 0 and k in _BULKY):
            continue
        out["ref_" + k] = v
    return out


def main(names=None):
    subprocess_ok = os.path.exists(pyoracle.REF_HARNESS)
    if not subprocess_ok:
        raise SystemExit("build the reference harness first: make -C oracle ref")
    todo = golden_cases()
    for name, (case, nsteps, stage, every) in todo.items():
        if names and name not in names:
            continue
        with tempfile.TemporaryDirectory() as tmp:
            base = case.write(tmp, name)
            ref = pyoracle.run_reference(base, nsteps, os.path.join(tmp, "out"), stage=stage, every=every,
                                         threads=1)
        payload = fixture_payload(case, ref, nsteps, stage)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **payload)
        print(f"{name}: {case.mesh.nelem} tets, {nsteps} steps -> {os.path.getsize(path) / 1024:.0f} KB")


def load_case(path: str):
    """Rebuilds the cases.Case stored in a fixture."""
    z = np.load(path)
    params = json.loads(bytes(z["params_json"]).decode())
    for k in ("cinf",):
        if k in params:
            params[k] = tuple(params[k])
    mats = {int(k): tuple(v) for k, v in json.loads(bytes(z["materials_json"]).decode()).items()}
    m = cases.Mesh(coord=z["coord"], intma=z["intma"], bfaces=z["bfaces"], lattice=None, shape=None,
                   mat_elem=z["mat_elem"])
    c = cases.Case(mesh=m, bc_map={int(a): int(b) for a, b in z["bc_map"]}, params=params, materials=mats)
    return c, z


if __name__ == "__main__":
    main(sys.argv[1:] or None)
