"""Failure detection on the GPU path, made on the host or by bounded device
waits: non-convergence, non-finite fields, invalid meshes and a device wait
that runs out of its spin limit.  No test faults, traps or hangs a GPU."""
import numpy as np
import pytest

from helpers import fixture_path, load_case

pytestmark = pytest.mark.gpu


def _gpu():
    from cbs3d import gpu
    return gpu


# every PCG kernel checks the same conditions: automatic, the two global-vector
# kernels (two reductions, single reduction) and the register single-reduction one
KERNELS = [0, 1, 4, 5]


@pytest.mark.parametrize("kernel", KERNELS)
def test_not_converged_reports_and_context_survives(kernel):
    case, _ = load_case(fixture_path("cav6j"))
    case.params["cg_max_iter"] = 2
    gpu = _gpu()
    c = gpu.Context(case, pcg_kernel=kernel)
    with pytest.raises(gpu.CBSError) as e:
        c.step(1)
    assert e.value.code == 2
    assert "failed to converge" in e.value.message
    u, p, t = c.fields()          # context still usable
    assert np.all(np.isfinite(u))


@pytest.mark.parametrize("kernel", KERNELS)
def test_nonfinite_velocity_is_reported(kernel):
    case, _ = load_case(fixture_path("cav6j"))
    gpu = _gpu()
    c = gpu.Context(case, pcg_kernel=kernel)
    u, p, t = c.fields()
    interior = 3 * 150
    u[interior] = np.nan
    c.upload(u, p, t)
    with pytest.raises(gpu.CBSError) as e:
        c.step(1)
    assert e.value.code == 4
    assert "invalid pressure residual" in e.value.message


def test_inverted_tetrahedron_rejected():
    case, _ = load_case(fixture_path("cav4"))
    case.mesh.intma = case.mesh.intma.copy()
    case.mesh.intma[5, [1, 2]] = case.mesh.intma[5, [2, 1]]
    gpu = _gpu()
    with pytest.raises(gpu.CBSError) as e:
        gpu.Context(case)
    assert e.value.code == 1
    assert "non-positive tetrahedron volume at element 6" in e.value.message


def test_device_wait_times_out_and_device_stays_usable():
    gpu = _gpu()
    assert gpu.selftest_wait_timeout(0) == 5
    case, _ = load_case(fixture_path("cav4"))
    c = gpu.Context(case)
    c.step(1)
