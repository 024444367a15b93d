"""Multi-GPU batching on the host: LPT sharding of instances by tet count and
the gather of per-instance metrics, as world_size-2 gloo ranks on the CPU
with a stand-in runner (no GPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def test_lpt_shard_properties():
    from cbs3d.batch import lpt_shard, shard_loads
    w = [384000, 6000, 96000, 200000, 55000, 300000, 10000, 130000, 7000]
    for n in (1, 2, 3, 4):
        s = lpt_shard(w, n)
        assert sorted(i for part in s for i in part) == list(range(len(w)))
        loads = shard_loads(w, s)
        # LPT bound: max load <= 4/3 OPT, and OPT >= max(total/n, max weight)
        assert max(loads) <= 4.0 / 3.0 * max(sum(w) / n, max(w)) + 1e-9
        assert s == lpt_shard(w, n)   # deterministic
    assert lpt_shard([5, 5], 3)[2] == []


def test_lpt_shard_of_the_cavity_batch():
    from cbs3d import cases
    from cbs3d.batch import lpt_shard, shard_loads
    w = [c.mesh.nelem for c in cases.cavity_batch(count=12, n_lo=3, n_hi=9)]
    loads = shard_loads(w, lpt_shard(w, 2))
    assert abs(loads[0] - loads[1]) <= max(w)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import sys
    import datetime
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "cbs-3d_b200"))
    import torch.distributed as dist
    from cbs3d import cases
    from cbs3d.batch import run_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    cs = cases.cavity_batch(count=7, n_lo=3, n_hi=8, seed=99)

    def fake_runner(mine, steps):
        return [{"nelem": c.mesh.nelem, "steps": steps, "rank": rank} for c in mine]

    out = run_sharded(cs, 4, rank, world, fake_runner, dist)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, out, [c.mesh.nelem for c in cs]))


def test_sharded_batch_gathers_every_instance_once():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict()
    for _ in procs:
        r, out, sizes = q.get(timeout=120)
        res[r] = (out, sizes)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[1][0] is None
    out, sizes = res[0]
    assert [m["instance"] for m in out] == list(range(7))
    assert [m["nelem"] for m in out] == sizes
    assert {m["rank"] for m in out} == {0, 1}
    assert all(m["steps"] == 4 for m in out)
