"""The allocation-free entry point cbs3d_convergence_norms_static.

It exists for callers that cannot call cudaMalloc (a process whose device
memory belongs to another allocator, or one that budgeted its device memory
up front); its only scratch is a file-scope device array shared by every
call.  This test feeds it device copies of a context's state and requires the
engine's own convergence measures bit for bit, on calls in a row: a
two-block conjugate-heat-transfer case with the energy equation on, then a
one-block cavity with the energy equation off and no temperature arrays (a
call that read the first call's leftover partials would differ), then the
first case again.  The file sorts last so that a run stopping at the first
failure has already run every other test."""
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


def _state(name):
    """A context one step in, its engine measures and device copies of the
    fields the entry point reads (temperature left out when it is off)."""
    import torch

    from cbs3d import gpu
    case, _ = load_case(fixture_path(name))
    ctx = gpu.Context(case)
    ctx.step(1)
    temp = case.params.get("temp_calc", 0) > 0
    dev = {n: torch.tensor(ctx.get(n), dtype=torch.float64, device="cuda")
           for n in FIELDS if temp or not n.startswith("temperature")}
    flags = torch.tensor(_node_flags(case), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    return ctx, dev, flags, int(temp)


def _call(fn, dev, flags, npoin, temp):
    ptr = [ctypes.c_void_p(dev[n].data_ptr()) if n in dev else None for n in FIELDS]
    hb = (ctypes.c_double * 15)()
    rc = fn(0, *ptr, ctypes.c_void_p(flags.data_ptr()), npoin, temp, hb)
    return rc, np.array(hb[:])


def test_static_scratch_norms_match_engine_on_calls_in_a_row():
    import torch
    fn = _entry()
    big = _state("cht")        # 315 nodes: two blocks of partials, energy on
    small = _state("cav4")     # 125 nodes: one block, energy off
    assert big[0].npoin > 256 >= small[0].npoin
    for ctx, dev, flags, temp in (big, small, big):
        want = ctx.get("hb")
        dev_before = torch.cuda.current_device()
        rc, hb = _call(fn, dev, flags, ctx.npoin, temp)
        assert rc == 0
        assert torch.cuda.current_device() == dev_before
        assert np.array_equal(hb, want), (hb, want)
        if not temp:
            assert np.all(hb[12:15] == 0.0)


def test_static_scratch_rejects_orphan_node():
    fn = _entry()
    ctx, dev, flags, temp = _state("cav4")
    flags[7] = 0                # a node that touches no element
    rc, _ = _call(fn, dev, flags, ctx.npoin, temp)
    assert rc == 1


def test_static_scratch_rejects_oversize():
    fn = _entry()
    hb = (ctypes.c_double * 15)()
    dummy = ctypes.c_void_p(16)   # never dereferenced: the size check comes first
    rc = fn(0, *([dummy] * 9), 2_097_153, 0, hb)
    assert rc == 1
