"""The measurement probes the benchmark states its rooflines with: reading a
buffer that fits in L2 is faster than reading one that does not, HBM reads
and copies land in the B200's range, and a grid all-reduce of the persistent
PCG kernel takes microseconds."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def _bw(nbytes, passes, mode):
    from cbs3d import gpu
    L = gpu.lib()
    L.cbs3d_probe_bandwidth.argtypes = [ctypes.c_int, ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_double)]
    v = ctypes.c_double()
    assert L.cbs3d_probe_bandwidth(0, nbytes, passes, mode, ctypes.byref(v)) == 0
    return v.value


def test_bandwidth_l2_above_hbm():
    l2r, hbmr = _bw(48 << 20, 200, 0), _bw(1 << 30, 10, 0)
    l2c, hbmc = _bw(24 << 20, 200, 1), _bw(1 << 30, 5, 1)
    print(f"read GB/s: L2 {l2r:.0f} HBM {hbmr:.0f}; copy GB/s: L2 {l2c:.0f} HBM {hbmc:.0f}")
    assert 3000.0 < hbmr < 9000.0 and 3000.0 < hbmc < 9000.0
    assert l2r > 1.2 * hbmr


def test_bad_probe_arguments_rejected():
    from cbs3d import gpu
    L = gpu.lib()
    L.cbs3d_probe_bandwidth.argtypes = [ctypes.c_int, ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_double)]
    v = ctypes.c_double()
    assert L.cbs3d_probe_bandwidth(0, 1 << 20, 1, 7, ctypes.byref(v)) == 1
    assert L.cbs3d_probe_bandwidth(0, 100, 1, 0, ctypes.byref(v)) == 1


def test_allreduce_latency():
    from cbs3d import gpu
    L = gpu.lib()
    L.cbs3d_probe_allreduce.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    us = ctypes.c_double()
    assert L.cbs3d_probe_allreduce(0, 2000, ctypes.byref(us)) == 0
    print(f"grid all-reduce: {us.value:.2f} us")
    assert 0.2 < us.value < 50.0
