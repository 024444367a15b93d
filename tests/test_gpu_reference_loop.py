"""The reference's own step loop running on the drop-in: the reference
harness built with the GPU pressure backend of INTEGRATION.md
(oracle/gpu_pressure_solver.inc, cbs_ref_gpu_harness) calls cbs3d_pcg_solve
in place of ConjugateGradient::solvePressure and otherwise runs the
reference's code.  On the 16^3 cavity (config 1, 500 steps) it reproduces
the reference-only run to 1e-10 relative L2 on u and p after every 100
steps, with PCG iteration counts within 2 of the reference's every step."""
import os
import tempfile

import numpy as np
import pytest

from helpers import fixture_path, load_case, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-10


def test_reference_loop_on_gpu_pressure_solver():
    from oracle import pyoracle
    if not os.path.exists(pyoracle.REF_GPU_HARNESS):
        pytest.fail("oracle/_ref/cbs_ref_gpu_harness is not built (make -C oracle ref)")
    case, z = load_case(fixture_path("c1_cavity16"))
    with tempfile.TemporaryDirectory() as tmp:
        base = case.write(tmp, "c1")
        out = pyoracle.run_reference(base, 500, os.path.join(tmp, "out"), every=100, threads=1, gpu_pressure=True)
    hist = out["history"].reshape(500, 21)
    ref = z["ref_history"].reshape(500, 21)
    assert np.all(np.abs(hist[:, 1] - ref[:, 1]) <= 2)
    assert np.all(hist[:, 4] <= case.params["relToler"])
    for s in range(100, 501, 100):
        eu = rel_l2(out[f"step{s}_unkno"], z[f"ref_step{s}_unkno"])
        ep = rel_l2(out[f"step{s}_pres"], z[f"ref_step{s}_pres"])
        print(f"step {s}: rel L2 u {eu:.2e} p {ep:.2e}")
        assert eu <= TOL and ep <= TOL
