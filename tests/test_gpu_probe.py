"""The measurement probes the benchmark states its rooflines with: the copy
bandwidth of an L2-resident buffer pair exceeds that of an HBM-sized pair,
and a grid all-reduce of the persistent PCG kernel takes microseconds."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def test_copy_bandwidth_l2_above_hbm():
    from cbs3d import gpu
    L = gpu.lib()
    L.cbs3d_probe_copy_bandwidth.argtypes = [ctypes.c_int, ctypes.c_longlong, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_double)]
    l2, hbm = ctypes.c_double(), ctypes.c_double()
    assert L.cbs3d_probe_copy_bandwidth(0, 24 << 20, 50, ctypes.byref(l2)) == 0
    assert L.cbs3d_probe_copy_bandwidth(0, 1 << 30, 5, ctypes.byref(hbm)) == 0
    print(f"copy GB/s: L2-resident {l2.value:.0f}, HBM {hbm.value:.0f}")
    assert 2000.0 < hbm.value < 9000.0
    assert l2.value > 1.2 * hbm.value


def test_allreduce_latency():
    from cbs3d import gpu
    L = gpu.lib()
    L.cbs3d_probe_allreduce.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    us = ctypes.c_double()
    assert L.cbs3d_probe_allreduce(0, 2000, ctypes.byref(us)) == 0
    print(f"grid all-reduce: {us.value:.2f} us")
    assert 0.2 < us.value < 50.0
