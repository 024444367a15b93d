"""The allocation-free entry point cbs3d_convergence_norms_static.

It exists for callers that cannot call cudaMalloc (a host loop that must not
stall the device, or a process whose device memory belongs to another
allocator); its only scratch is a file-scope device array.  This test feeds it
device copies of a context's state and compares its measures with the ones the
engine's own convergence kernels produced, on two calls in a row, so a second
call over the shared scratch must not see the first call's leftovers.  The
file sorts last so that a run stopping at the first failure has already run
every other test."""
import ctypes

import numpy as np
import pytest

from helpers import fixture_path, load_case

pytestmark = pytest.mark.gpu

FIELDS = ("unkno", "unkn1", "pres", "pres1", "temperature", "temperature1", "elcoe2", "elcoe2p")


def _entry():
    from cbs3d import gpu
    fn = gpu.lib().cbs3d_convergence_norms_static
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 9 + [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    return fn


def _node_flags(case) -> np.ndarray:
    m = case.mesh
    flags = np.zeros(m.npoin, dtype=np.uint8)
    fluid = m.mat_elem == 0
    flags[np.unique(m.intma[fluid] - 1)] |= 1
    flags[np.unique(m.intma[~fluid] - 1)] |= 2
    return flags


def test_static_scratch_norms_match_engine_on_two_calls():
    import torch

    from cbs3d import gpu
    case, _ = load_case(fixture_path("cht"))      # fluid + solid nodes, energy on
    ctx = gpu.Context(case)
    flags = torch.tensor(_node_flags(case), dtype=torch.uint8, device="cuda")
    fn = _entry()
    for _ in range(2):
        ctx.step(1)
        want = ctx.get("hb")
        dev = {n: torch.tensor(ctx.get(n), dtype=torch.float64, device="cuda") for n in FIELDS}
        torch.cuda.synchronize()
        hb = (ctypes.c_double * 15)()
        rc = fn(0, *[ctypes.c_void_p(dev[n].data_ptr()) for n in FIELDS], ctypes.c_void_p(flags.data_ptr()),
                ctx.npoin, 1, hb)
        assert rc == 0
        np.testing.assert_allclose(np.array(hb[:]), want, rtol=1e-12, atol=1e-300)


def test_static_scratch_rejects_oversize():
    fn = _entry()
    hb = (ctypes.c_double * 15)()
    dummy = ctypes.c_void_p(16)   # never dereferenced: the size check comes first
    rc = fn(0, *([dummy] * 9), 2_097_153, 0, hb)
    assert rc == 1
