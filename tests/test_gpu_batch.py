"""Batched step (cbs3d_batch_*, no reference counterpart): many independent
cases of uneven size advanced together, each instance's pressure system
solved with its own reductions and stopping test inside one cooperative
launch per wave.  Parity is per instance: against the reference's golden
vectors for the fixture cases, and against the single-case engine."""
import numpy as np
import pytest

from helpers import bitwise, fixture_path, load_case, rel_l2

pytestmark = pytest.mark.gpu

RUN_TOL = 1e-8       # short runs; solves differ from the single-case engine only in reduction grouping
MIXED_TOL = 1e-8


def _gpu():
    from cbs3d import gpu
    return gpu


def _fixtures(names):
    out = []
    for n in names:
        case, z = load_case(fixture_path(n))
        out.append((case, z))
    return out


def test_batch_fixtures_vs_reference():
    """Four fixture cases with three steps each -- cavity, CHT slab with
    materials and heat flux, global time step, mass-flow inlet with
    temperature -- batched; each matches the reference's golden vectors."""
    gpu = _gpu()
    fx = _fixtures(["cav4", "cht", "cav4_global", "chan_massflow"])
    b = gpu.Batch([c for c, _ in fx], autotune=False)
    stats, _ = b.step(3)
    for i, (case, z) in enumerate(fx):
        assert int(z["nsteps"][0]) == 3
        u, p, t = b.fields(i)
        assert rel_l2(u, z["ref_final_unkno"]) <= RUN_TOL
        assert rel_l2(p, z["ref_final_pres"]) <= RUN_TOL
        assert rel_l2(t, z["ref_final_temperature"]) <= RUN_TOL
        hist = z["ref_history"].reshape(3, 21)
        assert abs(stats[i].cg.iterations - int(hist[2, 1])) <= 2


def _uneven(count=6, seed=7):
    from cbs3d import cases
    return cases.cavity_batch(count=count, n_lo=4, n_hi=14, seed=seed, rel_tol=1e-10)


def test_batch_matches_single_contexts():
    """Uneven cavities (4..14 hexes per side, Re 50..1000): every instance of
    the batch agrees with the single-case engine run on its own."""
    gpu = _gpu()
    cs = _uneven()
    b = gpu.Batch(cs, autotune=False, rows_per_thread=2)
    bst, _ = b.step(6)
    for i, c in enumerate(cs):
        ctx = gpu.Context(c)
        st = ctx.step(6)
        u0, p0, _ = ctx.fields()
        u1, p1, _ = b.fields(i)
        assert rel_l2(u1, u0) <= RUN_TOL
        assert rel_l2(p1, p0) <= RUN_TOL
        assert abs(bst[i].cg.iterations - st.cg.iterations) <= 2
        ctx.close()


def test_batch_graph_and_eager_identical():
    gpu = _gpu()
    cs = _uneven(count=4, seed=11)
    runs = []
    for g in (True, False):
        b = gpu.Batch(cs, autotune=False, rows_per_thread=4, use_graph=g)
        b.step(2)
        b.step(3)
        runs.append([b.fields(i) for i in range(len(cs))])
        b.close()
    for a, c in zip(*runs):
        for x, y in zip(a, c):
            assert bitwise(x, y)


def test_batch_tilings_agree_and_autotuner_chooses_fastest():
    """Every tiling solves the same systems to the same tolerance; the
    autotuner times the feasible ones on the first step and keeps the
    fastest."""
    gpu = _gpu()
    cs = _uneven(count=5, seed=3)
    ref = None
    for rows, spread in ((2, 1), (8, 0)):
        b = gpu.Batch(cs, autotune=False, rows_per_thread=rows, spread=bool(spread))
        b.step(4)
        f = [b.fields(i) for i in range(len(cs))]
        if ref is None:
            ref = f
        else:
            for a, c in zip(ref, f):
                assert rel_l2(c[0], a[0]) <= RUN_TOL and rel_l2(c[1], a[1]) <= RUN_TOL
        b.close()
    b = gpu.Batch(cs, autotune=True)
    b.step(4)
    info = b.info()
    assert info["tuned"] == 1 and info["candidates"] >= 3
    timed = [(r, s, ms) for r, s, ms in info["candidates_timed"] if ms > 0]
    best = min(timed, key=lambda x: x[2])
    assert (info["rows_per_thread"], info["spread"]) == (best[0], best[1])
    for i, a in enumerate(ref):
        u, p, _ = b.fields(i)
        assert rel_l2(u, a[0]) <= RUN_TOL and rel_l2(p, a[1]) <= RUN_TOL


def test_batch_mixed_vs_fp64():
    """Mixed precision batch (FP32 inner PCG, FP64 defect correction) against
    the FP64 batch."""
    gpu = _gpu()
    cs = _uneven(count=4, seed=5)
    a = gpu.Batch(cs, autotune=False)
    a.step(5)
    m = gpu.Batch(cs, precision=gpu.MIXED, autotune=False)
    st, _ = m.step(5)
    assert m.info()["mixed_waves"] == 1
    for i in range(len(cs)):
        (u0, p0, _), (u1, p1, _) = a.fields(i), m.fields(i)
        assert rel_l2(u1, u0) <= MIXED_TOL and rel_l2(p1, p0) <= MIXED_TOL
        assert st[i].cg.outer_sweeps >= 1


def test_batch_rejects_bad_tiling():
    gpu = _gpu()
    with pytest.raises(gpu.CBSError):
        gpu.Batch(_uneven(count=2), autotune=False, rows_per_thread=3)


def test_engines_of_different_sizes_coexist():
    """A kernel's dynamic shared-memory limit is shared by every engine in
    the process: a small engine created after a large one must not break the
    large one's launches (single cases and batches alike)."""
    from cbs3d import cases
    gpu = _gpu()
    big = gpu.Context(cases.cavity(20, re=400.0, ntime=100, jitter=0.15, seed=1234))
    small = gpu.Context(cases.cavity(4, ntime=100))
    big.step(2)
    small.step(2)
    bb = gpu.Batch(_uneven(count=3, seed=1), autotune=False, rows_per_thread=8)
    bs = gpu.Batch(_uneven(count=2, seed=2), autotune=False, rows_per_thread=8)
    bb.step(2)
    bs.step(2)


def test_gpu_runner_drives_the_batch_on_one_device():
    """cbs3d.batch.run_sharded with the real gpu_runner on one GPU: every
    instance steps, and splitting the instances into the two LPT shards of a
    two-rank run (each shard its own batch, run one after the other here)
    gives every instance the PCG iteration counts of the single batch to
    within 2 (the CTAs an instance gets, and so its reduction order, depend on
    the batch it is packed with)."""
    from cbs3d import cases
    from cbs3d.batch import gpu_runner, lpt_shard, run_sharded
    cs = cases.cavity_batch(count=8, n_lo=4, n_hi=12)
    runner = gpu_runner(device=0)
    whole = run_sharded(cs, 3, 0, 1, runner)
    assert [m["instance"] for m in whole] == list(range(len(cs)))
    assert all(m["steps"] == 3 and m["cg_iterations"] > 0 for m in whole)
    shards = lpt_shard([c.mesh.nelem for c in cs], 2)
    assert all(shards)
    split = {}
    for part in shards:
        for i, m in zip(part, runner([cs[i] for i in part], 3)):
            split[i] = m
    for m in whole:
        assert abs(split[m["instance"]]["cg_iterations"] - m["cg_iterations"]) <= 2
        assert split[m["instance"]]["nelem"] == m["nelem"]
