"""Full-size configuration fixtures: the reference solver (oracle/_ref, built
from its own sources) runs the benchmark configurations at their full mesh
size for their stated step counts (64^3 cavity 200 steps, channel 200, CHT
slab 300), and a small fixture keeps what a GPU test needs to compare
against -- the generator call, a digest of the generated mesh, the per-step
history, whole-field norms and the fields at 4,000 seeded nodes, after every
EVERY-th step and at the end.

    make -C oracle ref && python tests/golden/make_config_golden.py [names]

At 8 host cores the 64^3 cavity takes about 10 s per reference step, so
its fixture is a one-off run of about 35 minutes.
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

# name -> (generator, kwargs, steps)
CONFIGS = {
    "cfg2_cavity64": ("cavity", dict(n=64, re=400.0, ntime=200, jitter=0.15, seed=1234), 200),
    "cfg4_channel": ("channel", dict(nx=96, ny=16, nz=16, length=6.0, re=100.0, ntime=200), 200),
    "cfg5_cht": ("cht_slab", dict(nx=128, ny_fluid=24, ny_solid=6, nz=24, length=4.0, re=200.0, pr=0.71,
                                  k_ratio=10.0, q=1.0, ntime=300), 300),
}
# sampled fields are kept after every EVERY-th step as well as at the end
EVERY = 50


def build(gen: str, kw: dict):
    return getattr(cases, gen)(**kw)


def mesh_digest(case) -> str:
    import hashlib
    h = hashlib.sha256()
    for a in (case.mesh.intma, case.mesh.coord, case.mesh.bfaces, case.mesh.mat_elem):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def sample_nodes(npoin: int) -> np.ndarray:
    return np.sort(np.random.default_rng(99).choice(npoin, size=min(4000, npoin), replace=False))


def main(names=None):
    if not os.path.exists(pyoracle.REF_HARNESS):
        raise SystemExit("build the reference harness first: make -C oracle ref")
    for name, (gen, kw, nsteps) in CONFIGS.items():
        if names and name not in names:
            continue
        case = build(gen, kw)
        with tempfile.TemporaryDirectory() as tmp:
            base = case.write(tmp, name)
            ref = pyoracle.run_reference(base, nsteps, os.path.join(tmp, "out"), every=EVERY,
                                         threads=os.cpu_count() or 1)
        idx = sample_nodes(case.mesh.npoin)
        u = ref["final_unkno"].reshape(-1, 3)
        snaps = list(range(EVERY, nsteps, EVERY))
        temp = case.params.get("temp_calc", 0) > 0
        out = {
            "generator": np.frombuffer(json.dumps({"gen": gen, "kw": kw}).encode(), dtype=np.uint8),
            "mesh_sha256": np.frombuffer(mesh_digest(case).encode(), dtype=np.uint8),
            "nsteps": np.array([nsteps], dtype=np.int32),
            "history": ref["history"],
            "idx": idx.astype(np.int32),
            "u": u[idx], "p": ref["final_pres"][idx], "t": ref["final_temperature"][idx],
            "norm_u": np.array([np.linalg.norm(u)]), "norm_p": np.array([np.linalg.norm(ref["final_pres"])]),
            "norm_t": np.array([np.linalg.norm(ref["final_temperature"])]),
            "snap_steps": np.array(snaps, dtype=np.int32),
        }
        for k in snaps:
            su = ref[f"step{k}_unkno"].reshape(-1, 3)
            sp = ref[f"step{k}_pres"]
            out[f"snap{k}_u"] = su[idx]
            out[f"snap{k}_p"] = sp[idx]
            out[f"snap{k}_norms"] = np.array([np.linalg.norm(su), np.linalg.norm(sp),
                                              np.linalg.norm(ref[f"step{k}_temperature"]) if temp else 0.0])
            if temp:
                out[f"snap{k}_t"] = ref[f"step{k}_temperature"][idx]
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **out)
        print(f"{name}: {case.mesh.nelem} tets, {nsteps} steps -> {os.path.getsize(path) / 1024:.0f} KB", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or None)
