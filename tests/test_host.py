"""Host-side checks that need no GPU: the C ABI library loads and exports
every entry point of include/cbs3d_gpu.h, the case-file reader, and the
synthetic case generator."""
import ctypes
import os
import re

import numpy as np
import pytest

from helpers import fixture_path, load_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_header_symbols():
    from cbs3d import gpu
    L = gpu.lib()
    hdr = open(os.path.join(ROOT, "include", "cbs3d_gpu.h")).read()
    names = set(re.findall(r"\b(cbs3d_[a-z_0-9]+)\s*\(", hdr))
    assert len(names) >= 20
    for n in sorted(names):
        assert hasattr(L, n), n


def test_read_params_matches_generated_par(tmp_path):
    from cbs3d import cases, gpu
    c = cases.cht_slab(4, 2, 2, 2, ntime=7, q=2.5)
    base = c.write(str(tmp_path), "x")
    par = gpu.Params()
    ne, npn, nb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    err = ctypes.create_string_buffer(512)
    rc = gpu.lib().cbs3d_read_params(base.encode(), ctypes.byref(par), ctypes.byref(ne), ctypes.byref(npn),
                                     ctypes.byref(nb), err, 512)
    assert rc == 0, err.value
    assert (ne.value, npn.value, nb.value) == (c.mesh.nelem, c.mesh.npoin, c.mesh.nboun)
    assert par.ntime == 7 and par.heat_flux_bc == 2.5 and par.temp_calc == 1
    assert par.material_properties_enabled == 1 and par.dimensional_mode == 1
    assert par.re == 200.0 and par.relToler == 1e-10 and par.cg_conv_test == 2
    assert par.steady_min_iterations == 7


def test_missing_case_is_io_error(tmp_path):
    from cbs3d import gpu
    with pytest.raises(gpu.CBSError) as e:
        gpu.Context(case_name=str(tmp_path / "nope"))
    assert e.value.code == 7


def test_unsupported_bco_id_rejected(tmp_path):
    from cbs3d import cases, gpu
    c = cases.cavity(2)
    c.bc_map[1] = 777
    base = c.write(str(tmp_path), "bad")
    with pytest.raises(gpu.CBSError) as e:
        gpu.Context(case_name=base)
    assert e.value.code == 1
    assert "unsupported solver BC ID 777" in e.value.message


def test_generator_shapes_and_orientation():
    from cbs3d import cases
    for c in (cases.cavity(5, jitter=0.15, seed=3), cases.channel(6, 2, 3), cases.cht_slab(6, 3, 2, 2)):
        m = c.mesh
        x = m.coord[m.intma - 1]
        v6 = np.einsum("ij,ij->i", x[:, 1] - x[:, 0], np.cross(x[:, 2] - x[:, 0], x[:, 3] - x[:, 0]))
        assert np.all(v6 > 0)
        nx, ny, nz = m.shape
        assert m.nelem == 6 * nx * ny * nz
        assert m.npoin == (nx + 1) * (ny + 1) * (nz + 1)
        assert m.nboun == 4 * (nx * ny + ny * nz + nx * nz)


def test_c2_sizes():
    from cbs3d import cases
    m = cases.box_mesh(64, 64, 64, jitter=0.15, seed=1234)
    assert (m.nelem, m.npoin, m.nboun) == (1572864, 274625, 49152)


def test_fixture_case_roundtrip():
    case, z = load_case(fixture_path("cht"))
    assert case.params["temp_calc"] == 1
    assert case.mesh.nelem == int(z["ref_sizes"][0])


def test_case_cache_round_trip(tmp_path):
    """The binary case cache returns exactly the parsed inputs, is reused
    while the source files are unchanged and is rebuilt when one changes."""
    import time
    from cbs3d import cases, gpu
    c = cases.cht_slab(6, 3, 2, 2, ntime=5)
    base = c.write(str(tmp_path), "cht")
    ref, hit = gpu.case_digest(base)
    assert not hit
    d1, hit1 = gpu.case_digest(base, use_cache=True)
    assert (d1, hit1) == (ref, False) and os.path.exists(base + ".cbscache")
    d2, hit2 = gpu.case_digest(base, use_cache=True)
    assert (d2, hit2) == (ref, True)
    time.sleep(0.01)
    with open(base + ".par", "a") as f:
        f.write("\n")
    d3, hit3 = gpu.case_digest(base, use_cache=True)
    assert not hit3 and d3 == ref


def test_case_cache_faster_on_large_mesh(tmp_path):
    import time
    from cbs3d import cases, gpu
    base = cases.cavity(28, ntime=5).write(str(tmp_path), "cav")
    t0 = time.perf_counter(); gpu.case_digest(base, use_cache=True); t_parse = time.perf_counter() - t0
    t0 = time.perf_counter(); _, hit = gpu.case_digest(base, use_cache=True); t_cache = time.perf_counter() - t0
    assert hit and t_cache < 0.5 * t_parse


def test_vtu_writer_layout(tmp_path):
    """The VTU carries the reference writer's arrays and cells: tets then
    boundary triangles, masks from the element materials, masked fields."""
    from cbs3d import cases, gpu
    from helpers import read_vtu
    c = cases.cht_slab(4, 2, 2, 2, ntime=3)
    base = c.write(str(tmp_path), "cht")
    N, E, NB = c.mesh.npoin, c.mesh.nelem, c.mesh.nboun
    rng = np.random.default_rng(0)
    u, p, t = rng.normal(size=3 * N), rng.normal(size=N), rng.normal(size=N)
    path = str(tmp_path / "x.vtu")
    err = ctypes.create_string_buffer(512)
    rc = gpu.lib().cbs3d_write_vtu_case(base.encode(), path.encode(), gpu._ptr(u), gpu._ptr(p), gpu._ptr(t), err, 512)
    assert rc == 0, err.value
    v = read_vtu(path)
    assert v["_npoints"] == N and v["_ncells"] == E + NB
    assert np.array_equal(v["Points"].reshape(-1), c.mesh.coord.reshape(-1))
    conn = v["connectivity"]
    assert np.array_equal(conn[:4 * E], (c.mesh.intma - 1).reshape(-1))
    assert np.array_equal(conn[4 * E:], (c.mesh.bfaces[:, :3] - 1).reshape(-1))
    assert np.array_equal(v["types"], np.r_[np.full(E, 10), np.full(NB, 5)])
    assert v["offsets"][-1] == 4 * E + 3 * NB
    mat = c.mesh.mat_elem
    tf = np.zeros(N, bool); ts = np.zeros(N, bool)
    for e in range(E):
        (tf if mat[e] == 0 else ts)[c.mesh.intma[e] - 1] = True
    assert np.array_equal(v["pressure_active"], tf.astype(np.int32))
    assert np.array_equal(v["velocity_active"], (tf & ~ts).astype(np.int32))
    assert np.array_equal(v["node_domain_kind"], np.where(tf & ts, 3, np.where(tf, 1, np.where(ts, 2, 0))))
    assert np.array_equal(v["pressure"], np.where(tf, p, 0.0))
    assert np.array_equal(v["temperature"], t)
    assert np.array_equal(v["velocity"], np.where((tf & ~ts)[:, None], u.reshape(-1, 3), 0.0))
    assert np.array_equal(v["mat_id"], np.r_[mat, np.full(NB, -1)])
    assert np.array_equal(v["cell_kind"], np.r_[np.full(E, 1), np.full(NB, 2)])
    assert np.array_equal(v["parent_element"][:E], np.arange(1, E + 1))


def test_abi_rejects_bad_inputs_before_touching_a_device():
    """Invalid sizes, connectivity and options are rejected on the host with
    the reference's messages (no device is needed to see them)."""
    from cbs3d import cases, gpu
    L = gpu.lib()
    c = cases.cavity(2, ntime=1)
    mesh, par, keep = gpu._mesh_params(c)
    opt = gpu.make_options()
    h = ctypes.c_void_p()
    err = ctypes.create_string_buffer(512)
    bad = gpu.Mesh(0, c.mesh.npoin, c.mesh.nboun, mesh.intma, mesh.coord, mesh.bface, mesh.mat_elem)
    assert L.cbs3d_create(ctypes.byref(bad), ctypes.byref(par), ctypes.byref(opt), ctypes.byref(h), err, 512) == 1
    assert b"non-positive mesh size" in err.value
    intma = c.mesh.intma.astype(np.int32).copy()
    intma[0, 0] = c.mesh.npoin + 5
    m2 = gpu.Mesh(c.mesh.nelem, c.mesh.npoin, c.mesh.nboun, gpu._ptr(intma), mesh.coord, mesh.bface, mesh.mat_elem)
    assert L.cbs3d_create(ctypes.byref(m2), ctypes.byref(par), ctypes.byref(opt), ctypes.byref(h), err, 512) == 1
    assert b"connectivity node out of range" in err.value
    assert L.cbs3d_create(None, ctypes.byref(par), ctypes.byref(opt), ctypes.byref(h), err, 512) == 1
    bo = gpu.BatchOptions()
    L.cbs3d_default_batch_options(ctypes.byref(bo))
    assert L.cbs3d_batch_create(0, None, None, ctypes.byref(bo), ctypes.byref(h), err, 512) == 1
    pcg = ctypes.c_void_p()
    assert L.cbs3d_pcg_create(c.mesh.nelem, c.mesh.npoin, gpu._ptr(intma), None, 0, None, None, None,
                              ctypes.byref(pcg), err, 512) == 1
    assert b"out of range" in err.value
    # a fixed-pressure node outside the fluid
    good = c.mesh.intma.astype(np.int32)
    bl = np.array([c.mesh.npoin + 1], dtype=np.int32)
    bv = np.zeros(1)
    assert L.cbs3d_pcg_create(c.mesh.nelem, c.mesh.npoin, gpu._ptr(good), None, 1, gpu._ptr(bl), gpu._ptr(bv), None,
                              ctypes.byref(pcg), err, 512) == 1
    assert b"fixed pressure node out of range" in err.value
    # the coarse-operator inverse checks its size and variant before any device call
    m = np.eye(3)
    out = np.empty_like(m)
    assert L.cbs3d_coarse_inverse(0, 0, gpu._ptr(m), gpu._ptr(out), 0) == 1
    assert L.cbs3d_coarse_inverse(0, 161, gpu._ptr(m), gpu._ptr(out), 0) == 1
    assert L.cbs3d_coarse_inverse(0, 165, gpu._ptr(m), gpu._ptr(out), 1) == 1
    assert L.cbs3d_coarse_inverse(0, 3, gpu._ptr(m), gpu._ptr(out), 2) == 1
    assert L.cbs3d_coarse_inverse(0, 3, None, gpu._ptr(out), 0) == 1


def test_parallel_section_parse_matches_sequential(tmp_path):
    """Large .plt files with one record per line are parsed by several
    threads; any other layout goes through the sequential scanner.  Both
    must give the same inputs and the same error for the same records."""
    from cbs3d import cases, gpu
    base = cases.cavity(32, ntime=5).write(str(tmp_path), "reg")   # 196,608 tets + 35,937 nodes
    plt = open(base + ".plt").read().split("\n")
    # the same records with the first element spread over two lines: sequential path
    alt = plt[:]
    first = alt[1].split()
    alt[1] = " ".join(first[:2]) + "\n" + " ".join(first[2:])
    alt_base = str(tmp_path / "alt")
    for ext in (".bco", ".par"):
        open(alt_base + ext, "w").write(open(base + ext).read())
    open(alt_base + ".plt", "w").write("\n".join(alt))
    d_par, _ = gpu.case_digest(base, use_cache=False)
    d_seq, _ = gpu.case_digest(alt_base, use_cache=False)
    assert d_par == d_seq
    # a node index out of range in element 1000, in both layouts
    for b, lines in ((base, plt), (alt_base, alt)):
        bad = lines[:]
        k = 1000 + (1 if b == alt_base else 0)
        t = bad[k].split()
        t[3] = str(10 ** 8)
        bad[k] = " ".join(t)
        open(b + ".plt", "w").write("\n".join(bad))
        with pytest.raises(gpu.CBSError) as e:
            gpu.case_digest(b, use_cache=False)
        assert "connectivity node out of range" in e.value.message


def test_bench_reference_arm_contract():
    """bench.py --impl reference times the reference's own OpenMP build on
    the host cores and prints the same metric with impl=reference."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if not os.path.exists(os.path.join(root, "oracle", "_ref", "cbs_ref_harness")):
        pytest.skip("reference harness not built")
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], cwd=root, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "steps/s"
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]


def test_integration_snippet_is_the_compiled_backend():
    """The solver_opt backend shown in INTEGRATION.md is the code that
    oracle/gpu_pressure_solver.inc compiles into the reference harness."""
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    doc = open(os.path.join(root, "INTEGRATION.md")).read()
    block = re.search(r"```cpp\n(.*?)```", doc, re.S).group(1)
    inc = open(os.path.join(root, "oracle", "gpu_pressure_solver.inc")).read()
    assert block.strip() in inc


def _gather_wavefronts(lc, slice_w, pos):
    """Half-warp bank-pair model of the neighbour gathers: per slot and half
    warp, the largest number of distinct halo entries sharing a bank pair."""
    w, off = 0, 0
    for width in slice_w:
        for u in range(width):
            for hw in range(2):
                p = {int(pos[lc[off + 32 * u + l]]) for l in range(16 * hw, 16 * hw + 16)}
                cnt = np.bincount(np.array(sorted(p)) % 16, minlength=16)
                w += max(1, int(cnt.max()))
        off += 32 * width
    return w


def test_halo_placement_probe():
    """The PCG engine's shared-memory placement of a CTA's halo (host only):
    a permutation that keeps every aligned block of 32 positions (so the
    staging loads read the same L2 sectors) and does not raise the gathers'
    bank-pair wavefronts; on random slot columns it lowers them.  The probe's
    wavefront counts match the model recomputed here."""
    from cbs3d import gpu
    L = gpu.lib()
    L.cbs3d_probe_halo_placement.restype = ctypes.c_int
    rng = np.random.default_rng(7)
    nh, widths = 1000, [12] * 20 + [9] * 12
    slice_w = np.array(widths, dtype=np.int32)
    slice_off = np.concatenate([[0], np.cumsum(32 * slice_w)]).astype(np.int64)
    lc = rng.integers(0, nh, size=int(slice_off[-1])).astype(np.uint16)
    pos = np.empty(nh, dtype=np.int32)
    wf = np.zeros(2, dtype=np.int64)
    P = ctypes.c_void_p
    rc = L.cbs3d_probe_halo_placement(nh, len(widths), P(slice_off.ctypes.data), P(slice_w.ctypes.data),
                                      P(lc.ctypes.data), P(pos.ctypes.data), P(wf.ctypes.data))
    assert rc == 0
    assert sorted(pos.tolist()) == list(range(nh))
    for b0 in range(0, nh, 32):
        assert set(pos[b0:b0 + 32].tolist()) == set(range(b0, min(nh, b0 + 32)))
    assert wf[0] == _gather_wavefronts(lc, widths, np.arange(nh))
    assert wf[1] == _gather_wavefronts(lc, widths, pos)
    assert wf[1] < wf[0]
    # a slot naming an entry past the halo is rejected
    bad = lc.copy()
    bad[5] = nh
    assert L.cbs3d_probe_halo_placement(nh, len(widths), P(slice_off.ctypes.data), P(slice_w.ctypes.data),
                                        P(bad.ctypes.data), P(pos.ctypes.data), P(wf.ctypes.data)) != 0
