"""Run output through the C++ host driver (cbs-3d_b200/cbs3d_run): the
residual CSV against the reference's per-step history for the same case,
and VTU/PVD snapshots against the engine's fields."""
import os
import subprocess

import numpy as np
import pytest

from helpers import bitwise, fixture_path, load_case, read_vtu

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "cbs-3d_b200", "cbs3d_run")
HEADER = ("iteration,time,dt,u_rel,u_norm,u_abs,v_rel,v_norm,v_abs,w_rel,w_norm,w_abs,p_rel,p_norm,p_abs,"
          "T_rel,T_norm,T_abs,velocity_rel_max,cg_iterations,cg_initial_l2,cg_final_l2,cg_relative_l2,cg_max_abs")


def test_driver_residual_csv_and_vtu(tmp_path):
    case, z = load_case(fixture_path("cav6j"))
    n = int(z["nsteps"][0])
    case.params.update(ntime=n, vtu=1, vtu_every=2, reslog=1, steady_min=n)
    base = case.write(str(tmp_path), "cav")
    r = subprocess.run([DRIVER, base, "--chunk", "3"], cwd=str(tmp_path), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = tmp_path / "output" / "cav"
    lines = (out / "cav_residuals.csv").read_text().splitlines()
    assert lines[0] == HEADER
    rows = np.array([[float(x) for x in l.split(",")] for l in lines[1:]])
    assert rows.shape == (n, 24)
    hist = z["ref_history"].reshape(n, 21)
    assert np.array_equal(rows[:, 0], np.arange(1, n + 1))
    assert np.allclose(rows[:, 2], hist[:, 0], rtol=1e-15, atol=0)              # dt, 16 digits
    assert np.all(np.abs(rows[:, 19] - hist[:, 1]) <= 2)                         # PCG iterations
    assert np.allclose(rows[:, 3:18], hist[:, 6:21], rtol=1e-6, atol=1e-14)     # Convergence::evaluate
    assert np.array_equal(rows[:, 18], np.maximum.reduce([rows[:, 3], rows[:, 6], rows[:, 9]]))
    names = sorted(os.listdir(out))
    vt = [f for f in names if f.endswith(".vtu")]
    assert vt == [f"cav_step_{k:08d}.vtu" for k in (0, 2, 4, 5)]
    pvd = (out / "cav.pvd").read_text()
    assert all(f'file="{f}"' in pvd for f in vt)
    from cbs3d import gpu
    ctx = gpu.Context(case)
    ctx.step(n)
    u, p, t = ctx.fields()
    v = read_vtu(str(out / vt[-1]))
    act = v["velocity_active"].astype(bool)
    assert bitwise(v["velocity"][act].reshape(-1), u.reshape(-1, 3)[act].reshape(-1))
    pa = v["pressure_active"].astype(bool)
    assert bitwise(v["pressure"][pa], p[pa])


def test_driver_reports_reference_errors(tmp_path):
    case, _ = load_case(fixture_path("cav4"))
    base = case.write(str(tmp_path), "bad")
    with open(base + ".bco") as f:
        txt = f.read()
    with open(base + ".bco", "w") as f:
        f.write(txt.replace("530", "777", 1))
    r = subprocess.run([DRIVER, base], cwd=str(tmp_path), capture_output=True, text=True, timeout=120)
    assert r.returncode == 1
    assert "unsupported solver BC ID 777" in r.stderr


def test_async_vtu_matches_immediate_vtu(tmp_path):
    """cbs3d_write_vtu_async gives the same file as cbs3d_write_vtu taken at
    the same point, although later steps are issued before it is written;
    three snapshots in a row exercise the wait for a free slot, and flush
    reports a file that cannot be written."""
    from cbs3d import gpu
    case, _ = load_case(fixture_path("cav6j"))
    ctx = gpu.Context(case)
    ctx.write_vtu(str(tmp_path / "s0.vtu"))
    ctx.write_vtu_async(str(tmp_path / "a0.vtu"))
    pairs = [("s0.vtu", "a0.vtu")]
    for k in (1, 2, 3):
        ctx.step(k)
        ctx.write_vtu(str(tmp_path / f"s{k}.vtu"))
        ctx.write_vtu_async(str(tmp_path / f"a{k}.vtu"))
        pairs.append((f"s{k}.vtu", f"a{k}.vtu"))
    ctx.step(2)   # issued while the last snapshots may still be copied out
    ctx.vtu_flush()
    for s, a in pairs:
        assert (tmp_path / s).read_bytes() == (tmp_path / a).read_bytes(), (s, a)
    ctx.write_vtu_async(str(tmp_path / "no_such_dir" / "x.vtu"))
    with pytest.raises(gpu.CBSError) as e:
        ctx.vtu_flush()
    assert e.value.code == 7 and "x.vtu" in e.value.message
    ctx.vtu_flush()   # the error is reported once
    ctx.write_vtu_async(str(tmp_path / "last.vtu"))
    ctx.close()       # writes what is pending
    assert (tmp_path / "last.vtu").stat().st_size > 0
