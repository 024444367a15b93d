#!/usr/bin/env python
"""CBS steps/s on the 64^3 jittered lid-driven cavity (1,572,864 P1 tets,
274,625 nodes, interior nodes jittered by U(-0.15h, 0.15h) from seed 1234,
Re=400, local time step csafm=0.5, Jacobi-PCG to relative 1e-10).

One "step" is one complete CBS step (time step, LHS, Steps 1-4, norms) on
device-resident state.  The timed region holds K steps bracketed by a
barrier and a device synchronise; time comes from CUDA events on the
engine's stream (max over ranks).  Every step streams ~0.9 GB of element
and node data, far more than the 126 MB L2, so no flush is inserted.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision both|fp64|mixed]
  python bench.py --impl reference ...   # the reference solver on the host cores

`value` is the FP64 engine with the reference's Jacobi-PCG (the drop-in for
the reference's FP64 path); with --precision both (the default) the same
line carries the mixed engine (FP32 inner PCG, FP64 defect correction) under
"mixed", the FP64 engine with the aggregation-multigrid preconditioner
(same stopping test) under "multigrid" and with the per-CTA two-level
preconditioner under "two_level": their steps/s and relative L2 errors on u
and p against the Jacobi FP64 engine after the same steps.  "batch" holds
the 48-cavity batched step (instance-steps/s, FP64 and mixed, against the
same instances stepped one after another).

Rooflines of the PCG kernel.  Bytes per iteration are the implemented
kernel's (the assembled SELL operator's coefficients and columns plus its
per-node vector traffic, cbs3d_step_stats.pcg_bytes_per_iter); the
element-by-element form's 64*E_f + 73*N (FP64) is reported beside them for
context only, since the assembled operator moves fewer bytes.  achieved =
bytes per iteration x iterations / the PCG launches' CUDA-event time.  At
64^3 the operator and vectors (~50 MB) stay in the 126 MB L2, so "roofline"
is stated against the L2 read bandwidth measured in this run (200 passes
over a 48 MiB buffer in one launch, cbs3d_probe_bandwidth; the PCG's L2
traffic is almost all reads), with the grid
all-reduce latency (cbs3d_probe_allreduce) as the per-iteration floor;
"hbm_case" runs the same FP64 engine on a 96^3 cavity, whose per-iteration
traffic exceeds L2 (the single-reduction global-vector kernel k_pcg64g),
against the HBM figure of MEASURED_PEAKS.json, else the 6,650 GB/s fallback
measured earlier on this pool (its source is stated in the line).

Multi-GPU: the single-case path does not shard (replicas only); each rank
runs its own replica and `value` is the total steps/s of all ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cbs-3d_b200"))
sys.path.insert(0, ROOT)

METRIC = "CBS steps/s, 64³ cavity: mixed vs FP64 GPU at ≤1e-8 rel err; PCG HBM GB/s"
N_HEX, RE, JITTER, SEED = 64, 400.0, 0.15, 1234


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"])
    ap.add_argument("--n", type=int, default=N_HEX, help="hexes per side")
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="cavity64", choices=["cavity64", "batch"],
                    help="batch: 48 seeded cavities of 10..40 hexes per side, Re 50..1000, batched step")
    ap.add_argument("--hbm-n", type=int, default=96, help="hexes per side of the HBM-bound PCG case (0: skip)")
    ap.add_argument("--hbm-steps", type=int, default=3)
    ap.add_argument("--batch-steps", type=int, default=10, help="timed steps of the batch key (0: skip)")
    return ap.parse_args()


def workload(n: int) -> str:
    return (f"lid-driven cavity {n}^3 hexes x 6 Kuhn tets, interior jitter +-{JITTER}h seed {SEED}, "
            f"Re={RE:g}, local dt csafm=0.5, Jacobi-PCG relTol 1e-10")


def make_case(n: int, ntime: int):
    from cbs3d import cases
    return cases.cavity(n, re=RE, ntime=ntime, jitter=JITTER, seed=SEED)


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
            return
        # nvidia-smi takes a few hundred ms to start: wait (at most 5 s) for its
        # first sample so that the samples cover the timed region
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.p.poll() is None and os.path.getsize(self.f.name) == 0:
            time.sleep(0.02)

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def probes(device: int) -> dict:
    """L2 and HBM read and copy bandwidths and the grid all-reduce latency on
    this GPU, measured with the library's probe kernels (CUDA events)."""
    import ctypes

    from cbs3d import gpu
    L = gpu.lib()
    L.cbs3d_probe_bandwidth.argtypes = [ctypes.c_int, ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_double)]
    L.cbs3d_probe_allreduce.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    out = {}
    for key, nbytes, passes, mode in (("l2_read_gbs", 48 << 20, 200, 0), ("l2_copy_gbs", 24 << 20, 200, 1),
                                      ("hbm_read_gbs", 1 << 30, 10, 0), ("hbm_copy_gbs", 1 << 30, 5, 1)):
        v = ctypes.c_double()
        if L.cbs3d_probe_bandwidth(device, nbytes, passes, mode, ctypes.byref(v)) == 0:
            out[key] = v.value
    ar = ctypes.c_double()
    if L.cbs3d_probe_allreduce(device, 4000, ctypes.byref(ar)) == 0:
        out["allreduce_us"] = ar.value
    return out


def ncu_traffic(kernel: str, n: int, its_per_launch: float):
    """DRAM bytes (read + write) of one PCG launch: the committed ncu figure
    per iteration for this kernel and mesh size (profiles/pcg_traffic.json)
    times this run's iterations per launch; None without a capture."""
    path = os.path.join(ROOT, "profiles", "pcg_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    per_it = d.get(kernel, {}).get(str(n))
    return None if per_it is None else per_it * its_per_launch


# ----------------------------------------------------------- CPU baseline
def reference_harness():
    return os.path.join(ROOT, "oracle", "_ref", "cbs_ref_harness")


def run_reference(case, steps: int, warmup: int, threads: int) -> dict:
    with tempfile.TemporaryDirectory() as tmp:
        base = case.write(tmp, "cavity")
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close", OMP_PLACES="cores")
        out = subprocess.run([reference_harness(), base, str(steps), tmp, "--time", "--warmup", str(warmup)],
                             check=True, capture_output=True, text=True, env=env)
    return json.loads(out.stdout.strip().splitlines()[-1])


def cpu_baseline(n: int) -> dict:
    threads = os.cpu_count() or 1
    if not os.path.exists(reference_harness()):
        return {"value": None, "unit": "steps/s", "cores": threads, "kind": "reference",
                "sample": "unavailable: oracle/_ref/cbs_ref_harness not built"}
    # the first three CBS steps (about 12 s on 16 host cores at 64^3)
    case = make_case(n, ntime=4)
    r = run_reference(case, steps=3, warmup=0, threads=threads)
    return {"value": r["steps_per_s"], "unit": "steps/s", "cores": r["threads"], "kind": "reference",
            "sample": f"first {r['steps']} CBS steps of the same {n}^3 cavity ({r['last_cg_iterations']} PCG "
                      f"iterations in the last), reference compiled from its sources, OpenMP {r['threads']} "
                      f"threads, {r['seconds']:.1f} s"}


# ----------------------------------------------------------------- arms
def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group(backend="nccl", timeout=datetime.timedelta(seconds=120))
    return ws, rank, local, dist


def dist_max(dist, x: float) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def arm_reference(args):
    ws, rank, _, dist = dist_init()
    if rank != 0:
        barrier(dist)
        if dist is not None:
            dist.destroy_process_group()
        return
    case = make_case(args.n, ntime=10 ** 6)
    threads = os.cpu_count() or 1
    # the requested steps, up to 20 timed after up to 5 warm-up steps (about
    # 4-5 s each on 16 host cores at 64^3), so the run ends within minutes
    k = max(1, min(args.steps, 20))
    w = min(args.warmup, 5)
    if not os.path.exists(reference_harness()):
        print(json.dumps({"impl": "reference", "unavailable": "reference harness oracle/_ref not built"}))
    else:
        r = run_reference(case, steps=k, warmup=w, threads=threads)
        v = r["steps_per_s"]
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": ws,
            "steps": r["steps"], "warmup": w, "ms_per_step": 1e3 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload(args.n), "precision": "fp64", "parallelism": "host OpenMP"},
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": r["threads"], "kind": "reference",
                             "sample": f"{r['steps']} timed CBS steps after {w} warm-up step(s) of the same "
                                       f"cavity; the reference's own OpenMP build ({r['threads']} threads)"},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
    barrier(dist)
    if dist is not None:
        dist.destroy_process_group()


def ebe_bytes(nelem_fluid: int, npoin: int, mixed: bool) -> int:
    """Bytes one PCG iteration of the element-by-element form would move:
    per fluid tet 4 int32 connectivity + 6 coefficients, per node p, Ap
    (written and read), pres and r (read and written), pdiag, new p, plus a
    one-byte mask -- FP64 64*E_f + 73*N, FP32 inner 40*E_f + 37*N."""
    return (40 * nelem_fluid + 37 * npoin) if mixed else (64 * nelem_fluid + 73 * npoin)


KERNELS = {1: "k_pcg64", 2: "k_pcg64r", 3: "k_pcg64h", 4: "k_pcg64c", 5: "k_pcg32m", 6: "k_pcg64d", 7: "k_pcg_mg",
           8: "k_pcg64g", 9: "k_pcg64c"}


def timed_run(args, ctx, dist):
    """W warm-up steps, then K steps between barriers; returns the stats of
    both calls, the max-over-ranks device seconds and the clocks seen."""
    warm = ctx.step(args.warmup)
    clocks = ClockSampler(ctx.device)
    barrier(dist)
    st = ctx.step(args.steps)
    barrier(dist)
    sec = dist_max(dist, st.gpu_seconds)
    return warm, st, sec, clocks.stop()


def roofline(st, warm, nelem_fluid, npoin, mixed, n, pr, bound="l2"):
    """PCG kernel roofline: the kernel's own bytes per iteration over its
    CUDA-event time, against the L2 read bandwidth measured in this run
    (bound "l2": the solve's operator and vectors stay in L2) or the HBM
    figure (bound "hbm": MEASURED_PEAKS.json, else the fallback)."""
    hbm, hbm_kind = measured_peak()
    its = st.cg_iterations_total - warm.cg_iterations_total   # totals are cumulative
    kb = float(st.pcg_bytes_per_iter)
    achieved = its * kb / st.pcg_seconds / 1e9 if st.pcg_seconds > 0 and its > 0 else None
    kname = KERNELS.get(st.pcg_kernel, "?")
    if bound == "l2":
        peak = pr.get("l2_read_gbs")
        src = ("measured in this run: 200 read passes over a 48 MiB L2-resident buffer in one launch "
               "(cbs3d_probe_bandwidth, CUDA events)")
    else:
        peak, src = hbm, hbm_kind
    out = {"bound": bound, "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": achieved / peak if achieved and peak else None,
           "traffic": ncu_traffic(kname, n, its / max(st.pcg_launches, 1)),
           "traffic_unit": "DRAM bytes per launch (one pressure solve): ncu bytes per iteration x this run's "
                           "iterations per launch",
           "kernel": f"{kname} (persistent PCG, one launch per pressure solve)", "peak_source": src,
           "kernel_bytes_per_iteration": kb, "ebe_bytes_per_iteration": ebe_bytes(nelem_fluid, npoin, mixed),
           "iterations": its, "us_per_iteration": 1e6 * st.pcg_seconds / its if its > 0 else None,
           "launches": st.pcg_launches, "avg_launch_ms": 1e3 * st.pcg_seconds / max(st.pcg_launches, 1)}
    if st.pcg_kernel == 9:
        out["operator_storage"] = ("SELL coefficients held on chip in the SM's tensor memory for the whole solve "
                                   "(tcgen05.ld every iteration); kernel_bytes_per_iteration still counts them, "
                                   "with the vectors, as the algorithm's bytes")
    if bound == "l2":
        out["hbm_peak"] = hbm
        out["hbm_peak_source"] = hbm_kind
        out["hbm_frac"] = achieved / hbm if achieved else None
        out["allreduce_us"] = pr.get("allreduce_us")
    return out


def hbm_case(args, local, dist):
    """The FP64 Jacobi engine on a cavity whose PCG traffic per iteration
    exceeds L2 (96^3 by default): the PCG roofline against HBM."""
    from cbs3d import gpu
    n = args.hbm_n
    case = make_case(n, ntime=10 ** 6)
    ctx = gpu.Context(case, precision=gpu.FP64, device=local, use_graph=False, time_pcg=True)
    warm = ctx.step(1)
    barrier(dist)
    st = ctx.step(args.hbm_steps)
    barrier(dist)
    sec = dist_max(dist, st.gpu_seconds)
    roof = roofline(st, warm, case.mesh.nelem, ctx.npoin, False, n, {}, bound="hbm")
    ctx.close()
    roof.update({"workload": workload(n), "nelem": case.mesh.nelem, "npoin": case.mesh.npoin,
                 "steps": args.hbm_steps, "steps_per_s": args.hbm_steps / sec,
                 "pcg_share_of_step": st.pcg_seconds / st.gpu_seconds if st.gpu_seconds > 0 else None})
    return roof


def batch_key(args, local, dist):
    """The 48-cavity batch (pressure solves to 1e-8), FP64 and mixed, against
    the same instances stepped one after another on single contexts."""
    from cbs3d import cases, gpu
    cs = cases.cavity_batch()
    out = {"workload": "48 lid-driven cavities, 10..40 hexes per side x 6 Kuhn tets, Re log-uniform 50..1000, "
                       "seed 2024, Jacobi-PCG relTol 1e-8, one batched step per CUDA graph",
           "instances": len(cs), "nelem_total": int(sum(c.mesh.nelem for c in cs)), "steps": args.batch_steps,
           "unit": "instance-steps/s"}
    for name, prec in (("fp64", gpu.FP64), ("mixed", gpu.MIXED)):
        b = gpu.Batch(cs, precision=prec, device=local, autotune=True)
        b.step(max(args.warmup, 1))            # the autotuner runs in the first step
        barrier(dist)
        st, sec = b.step(args.batch_steps)
        barrier(dist)
        sec = dist_max(dist, sec)
        out[name] = {"value": len(cs) * args.batch_steps / sec, "ms_per_step": 1e3 * sec / args.batch_steps,
                     "autotuned": b.info(), "gpu_launches": int(sum(x.kernel_launches for x in st))}
        b.close()
    seq = 0.0
    for c in cs:
        ctx = gpu.Context(c, precision=gpu.FP64, device=local)
        ctx.step(1)
        seq += ctx.step(args.batch_steps).gpu_seconds
        ctx.close()
    out["sequential_fp64_ms_per_step"] = 1e3 * seq / args.batch_steps
    out["speedup_fp64_vs_sequential"] = out["sequential_fp64_ms_per_step"] / out["fp64"]["ms_per_step"]
    out["mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def arm_gpu(args):
    from cbs3d import gpu
    ws, rank, local, dist = dist_init()
    case = make_case(args.n, ntime=10 ** 6)
    nelem_fluid = case.mesh.nelem          # the cavity is all fluid
    first = gpu.MIXED if args.precision == "mixed" else gpu.FP64
    pr = probes(local)
    ctx = gpu.Context(case, precision=first, device=local, use_graph=False, time_pcg=True)
    N = ctx.npoin
    warm, st, sec, clk = timed_run(args, ctx, dist)
    value = ws * args.steps / sec
    roof = roofline(st, warm, nelem_fluid, N, first == gpu.MIXED, args.n, pr)
    u0, p0, _ = ctx.fields()

    # end to end through the public API with host buffers: upload the state,
    # one step, download the state, every step
    e2e = None
    if args.e2e_steps > 0:
        import torch
        pin = torch.empty(5 * N, dtype=torch.float64, pin_memory=True).numpy()
        u, p, t = ctx.fields()
        pin[:3 * N] = u
        pin[3 * N:4 * N] = p
        pin[4 * N:] = t
        hu, hp, ht = pin[:3 * N], pin[3 * N:4 * N], pin[4 * N:]
        barrier(dist)
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            ctx.upload(hu, hp, ht)
            ctx.step(1)
            ctx._check(gpu.lib().cbs3d_download_fields(ctx.h, gpu._ptr(hu), gpu._ptr(hp), gpu._ptr(ht)))
        el = dist_max(dist, time.perf_counter() - t0)
        e2e = {"value": ws * args.e2e_steps / el, "unit": "steps/s", "h2d_bytes_per_step": 5 * N * 8,
               "d2h_bytes_per_step": 5 * N * 8}
    launches = int(st.kernel_launches)
    its_per_step = roof["iterations"] / args.steps
    pcg_share = st.pcg_seconds / st.gpu_seconds if st.gpu_seconds > 0 else None
    ctx.close()

    def fp64_variant(**kw):
        vctx = gpu.Context(case, precision=gpu.FP64, device=local, use_graph=False, time_pcg=True, **kw)
        vwarm, vst, vsec, _ = timed_run(args, vctx, dist)
        uv, pv, _ = vctx.fields()
        out = {"value": ws * args.steps / vsec, "unit": "steps/s", "ms_per_step": 1e3 * vsec / args.steps,
               "speedup_vs_fp64": (ws * args.steps / vsec) / value, "pcg_kernel": int(vst.pcg_kernel),
               "rel_l2_u_vs_fp64": float(np.linalg.norm(uv - u0) / np.linalg.norm(u0)),
               "rel_l2_p_vs_fp64": float(np.linalg.norm(pv - p0) / np.linalg.norm(p0)),
               "pcg_iterations_per_step": (vst.cg_iterations_total - vwarm.cg_iterations_total) / args.steps,
               "pcg_share_of_step": vst.pcg_seconds / vst.gpu_seconds if vst.gpu_seconds > 0 else None,
               "gpu_launches": int(vst.kernel_launches),
               "roofline": roofline(vst, vwarm, nelem_fluid, N, False, args.n, pr)}
        vctx.close()
        return out

    # the aggregation-multigrid preconditioner (extension): FP64, same stopping test
    mgk = fp64_variant(multigrid=True) if args.precision in ("both", "fp64") else None

    # the two-level preconditioner (extension): FP64, same stopping test
    two = None
    if args.precision in ("both", "fp64"):
        tctx = gpu.Context(case, precision=gpu.FP64, device=local, use_graph=False, time_pcg=True, two_level=True)
        twarm, tst, tsec, _ = timed_run(args, tctx, dist)
        ut, pt, _ = tctx.fields()
        two = {"value": ws * args.steps / tsec, "unit": "steps/s", "ms_per_step": 1e3 * tsec / args.steps,
               "speedup_vs_fp64": (ws * args.steps / tsec) / value, "pcg_kernel": int(tst.pcg_kernel),
               "rel_l2_u_vs_fp64": float(np.linalg.norm(ut - u0) / np.linalg.norm(u0)),
               "rel_l2_p_vs_fp64": float(np.linalg.norm(pt - p0) / np.linalg.norm(p0)),
               "pcg_iterations_per_step": (tst.cg_iterations_total - twarm.cg_iterations_total) / args.steps}
        two["gpu_launches"] = int(tst.kernel_launches)
        tctx.close()

    mixed = None
    if args.precision == "both":
        mctx = gpu.Context(case, precision=gpu.MIXED, device=local, use_graph=False, time_pcg=True)
        mwarm, mst, msec, _ = timed_run(args, mctx, dist)
        um, pm, _ = mctx.fields()
        mixed = {"value": ws * args.steps / msec, "unit": "steps/s", "ms_per_step": 1e3 * msec / args.steps,
                 "speedup_vs_fp64": (ws * args.steps / msec) / value,
                 "rel_l2_u_vs_fp64": float(np.linalg.norm(um - u0) / np.linalg.norm(u0)),
                 "rel_l2_p_vs_fp64": float(np.linalg.norm(pm - p0) / np.linalg.norm(p0)),
                 "pcg_iterations_per_step": (mst.cg_iterations_total - mwarm.cg_iterations_total) / args.steps,
                 "roofline": roofline(mst, mwarm, nelem_fluid, N, True, args.n, pr)}
        mixed["gpu_launches"] = int(mst.kernel_launches)
        mctx.close()

    hbm = hbm_case(args, local, dist) if args.hbm_n > 0 else None
    bat = batch_key(args, local, dist) if args.batch_steps > 0 else None

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.n)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if first == gpu.FP64 else "f32+f64",
            "data": "synthetic",
            "config": {"workload": workload(args.n), "nelem": case.mesh.nelem, "npoin": N,
                       "precision": "fp64" if first == gpu.FP64 else "mixed",
                       "l2": "inputs larger than L2 (no flush): each step streams the element arrays, "
                             "about 0.6 GB at 64^3",
                       "parallelism": "replicas" if ws > 1 else "single"},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk,
            "pcg_iterations_per_step": its_per_step, "pcg_share_of_step": pcg_share, "probes": pr,
        }
        if mixed is not None:
            line["mixed"] = mixed
        if mgk is not None:
            line["multigrid"] = mgk
        if two is not None:
            line["two_level"] = two
        if hbm is not None:
            line["hbm_case"] = hbm
        if bat is not None:
            line["batch"] = bat
        print(json.dumps(line))
    if dist is not None:
        barrier(dist)
        dist.destroy_process_group()


def arm_batch(args):
    """Batched step on 48 uneven cavities (pressure solves to 1e-8): the
    instances are LPT-sharded by tet count over the ranks; value = instance
    steps per second of the whole job."""
    from cbs3d import cases, gpu
    from cbs3d.batch import lpt_shard
    ws, rank, local, dist = dist_init()
    cs = cases.cavity_batch()
    shards = lpt_shard([c.mesh.nelem for c in cs], ws)
    mine = [cs[i] for i in shards[rank]]
    prec = gpu.MIXED if args.precision == "mixed" else gpu.FP64
    b = gpu.Batch(mine, precision=prec, device=local, autotune=True)
    b.step(max(args.warmup, 1))            # the autotuner runs in the first step
    clocks = ClockSampler(local)
    barrier(dist)
    st, sec = b.step(args.steps)
    barrier(dist)
    sec = dist_max(dist, sec)
    clk = clocks.stop()
    info = b.info()
    launches = int(sum(x.kernel_launches for x in st))
    b.close()
    # the same batch with FP32 inner solves and FP64 residual replacement
    # (the batched configuration's solver), timed the same way
    mixed = None
    if args.precision == "both":
        bm = gpu.Batch(mine, precision=gpu.MIXED, device=local, autotune=True)
        bm.step(max(args.warmup, 1))
        barrier(dist)
        mst, msec = bm.step(args.steps)
        barrier(dist)
        msec = dist_max(dist, msec)
        mixed = {"value": len(cs) * args.steps / msec, "unit": "instance-steps/s",
                 "ms_per_step": 1e3 * msec / args.steps, "speedup_vs_fp64": sec / msec,
                 "batch_rank0": bm.info(), "gpu_launches": int(sum(x.kernel_launches for x in mst))}
        bm.close()
    if rank == 0:
        print(json.dumps({
            "metric": "CBS instance-steps/s, 48 batched cavities", "value": len(cs) * args.steps / sec,
            "unit": "instance-steps/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sec / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64" if prec == gpu.FP64 else "f32+f64", "data": "synthetic",
            "config": {"workload": "48 lid-driven cavities, 10..40 hexes per side x 6 Kuhn tets, Re log-uniform "
                                   "50..1000, seed 2024, Jacobi-PCG relTol 1e-8, one batched step per CUDA graph",
                       "nelem_total": int(sum(c.mesh.nelem for c in cs)), "parallelism": f"LPT shards x{ws}",
                       "l2": "inputs larger than L2 (no flush)"},
            "batch_rank0": info, "gpu_launches": launches, "clocks": clk, "mixed": mixed}))
    if dist is not None:
        barrier(dist)
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "gpu" and args.workload == "batch":
        arm_batch(args)
        return
    if args.impl == "reference":
        arm_reference(args)
    else:
        arm_gpu(args)


if __name__ == "__main__":
    main()
