"""GPU path against the reference's golden vectors and the oracle, through
the C ABI (libcbs3d_gpu.so).

Bitwise: preprocessing, colouring, BC lists, time step, LHS diagonals,
Step 1, Step-2 RHS, the colour-ordered matvec, Step 3 and Step 4 (each stage
fed the reference's inputs).  Tolerance: the PCG solve, whose dot products
and assembled-operator sums run in a different (deterministic) order than
the reference's serial loops -- every solve meets the reference's own
stopping test ||r||/||r0|| <= relToler, and solutions agree to
PCG_TOL relative L2; multi-step runs agree to RUN_TOL."""
import json

import numpy as np
import pytest

from helpers import STAGED, bitwise, fixture_path, load_case, rel_l2, stage_step

pytestmark = pytest.mark.gpu

PCG_TOL = 1e-8       # one pressure solve to relToler=1e-10, vs the reference's
RUN_TOL = 1e-8       # short multi-step runs
C1_TOL = 1e-10       # config-1 cavity after 500 steps (u, p)
PRE = ["fedge", "detJ", "dNkdx", "annxf", "alen_e", "pdiagE", "gstifE", "color_ptr", "color_elem",
       "bc_list", "bc_values", "wall_node_list", "face_norm", "iside"]


def _gpu():
    from cbs3d import gpu
    return gpu


def _ctx(name, **kw):
    case, z = load_case(fixture_path(name))
    return _gpu().Context(case, **kw), case, z


def _param(z, key):
    return json.loads(bytes(z["params_json"]).decode()).get(key, 0)


@pytest.mark.parametrize("name", STAGED)
def test_preprocess_bitwise(name):
    c, _, z = _ctx(name)
    for k in PRE:
        assert bitwise(c.get(k), z["ref_" + k]), k
    u, p, t = c.fields()
    assert bitwise(u, z["ref_init_unkno"])
    assert bitwise(p, z["ref_init_pres"])
    assert bitwise(t, z["ref_init_temperature"])
    assert bitwise(c.get("Mdiag_real"), z["ref_Mdiag_real"])


@pytest.mark.parametrize("name", STAGED)
def test_stages_bitwise(name):
    c, _, z = _ctx(name)
    k = stage_step(z)
    for _ in range(k - 1):
        c.stage("begin_step")   # advance the step counter only
    c.upload(z["ref_s0_unkno"], z["ref_s0_pres"], z["ref_s0_temperature"])
    c.stage("begin_step")
    c.stage("time_step")
    assert bitwise(c.get("delte"), z["ref_s1_delte"])
    assert bitwise(c.get("dtreal"), z["ref_s1_dtreal"])
    c.stage("lhs")
    for a in ("elcoe2", "elcoe2p", "pdiag", "gstif", "pres"):
        assert bitwise(c.get(a), z["ref_s2_" + a]), a
    c.stage("step1")
    assert bitwise(c.get("rhs"), z["ref_s3_rhs"])
    assert bitwise(c.get("unkno"), z["ref_s3_unkno"])
    if _param(z, "step2_check"):
        c.stage("dt_correction")
        c.stage("lhs")
    c.stage("step2_rhs")
    assert bitwise(c.get("rhs1"), z["ref_s4_rhs1"])
    assert bitwise(c.get("pdiag"), z["ref_s4_pdiag_in"])
    assert bitwise(c.get("gstif"), z["ref_s4_gstif"])
    # MatrixVectorCalc::pressureMultiply in colour order
    assert bitwise(c.pressure_multiply(z["ref_s4_pres_in"]), z["ref_s4_Apres"])
    c.stage("solve_pressure")
    cg = c.get("cg")
    assert rel_l2(c.get("pres"), z["ref_s5_pres"]) <= PCG_TOL
    assert abs(int(cg[0]) - int(z["ref_s5_cg"][0])) <= 2
    assert bitwise(c.get("rhs1"), z["ref_s5_rhs1"])
    assert bitwise(c.get("pdiag"), z["ref_s5_pdiag"])
    # Step 3/4 from the reference's pressure
    c.set("pres", z["ref_s5_pres"])
    c.stage("step3")
    assert bitwise(c.get("rhs"), z["ref_s6_rhs"])
    assert bitwise(c.get("unkno"), z["ref_s6_unkno"])
    c.stage("step4")
    if "ref_s7_temperature" in z.files:
        assert bitwise(c.get("rhs1"), z["ref_s7_rhs1"])
        assert bitwise(c.get("temperature"), z["ref_s7_temperature"])
    c.stage("convergence")
    assert bitwise(c.get("velocity"), z["ref_s8_velocity"])
    np.testing.assert_allclose(c.get("hb"), z["ref_s8_hb"], rtol=1e-12, atol=1e-300)


@pytest.mark.parametrize("name", STAGED)
def test_full_run(name):
    c, _, z = _ctx(name)
    n = int(z["nsteps"][0])
    hist = z["ref_history"].reshape(n, 21)
    for s in range(n):
        st = c.step(1)
        assert abs(st.cg.iterations - int(hist[s, 1])) <= 2
        assert abs(st.dtreal - hist[s, 0]) <= 1e-12 * abs(hist[s, 0])
    u, p, t = c.fields()
    assert rel_l2(u, z["ref_final_unkno"]) <= RUN_TOL
    assert rel_l2(p, z["ref_final_pres"]) <= RUN_TOL
    if _param(z, "temp_calc") or _param(z, "material_enabled"):
        assert rel_l2(t, z["ref_final_temperature"]) <= RUN_TOL


def test_c1_cavity16_500_steps():
    """Config 1: 16^3 x 6 Kuhn cavity, Re=100, local dt csafm=0.5,
    Jacobi-PCG relTol 1e-10, 500 steps; u and p within 1e-10 relative L2 of
    the reference after every 100 steps."""
    c, _, z = _ctx("c1_cavity16")
    hist = z["ref_history"].reshape(500, 21)
    for blk in range(5):
        st = c.step(100)
        s = (blk + 1) * 100
        u, p, _ = c.fields()
        eu = rel_l2(u, z[f"ref_step{s}_unkno"])
        ep = rel_l2(p, z[f"ref_step{s}_pres"])
        print(f"step {s}: rel L2 u {eu:.3e} p {ep:.3e} cg {st.cg.iterations} (ref {int(hist[s - 1, 1])})")
        assert eu <= C1_TOL and ep <= C1_TOL
    assert abs(st.cg.iterations - int(hist[-1, 1])) <= 2


def test_dropin_pressure_solver():
    """cbs3d_pcg_solve with the reference's Step-2 inputs (solver_opt=1 drop-in)."""
    case, z = load_case(fixture_path("cav6j"))
    gpu = _gpu()
    bc_list = z["ref_bc_list"]
    ps = gpu.PressureSolver(case.mesh.intma, case.mesh.mat_elem, bc_list, z["ref_bc_values"])
    pres, rhs1, pdiag, res = ps.solve(z["ref_s4_gstif"], z["ref_s4_pdiag_in"], z["ref_s4_rhs1"],
                                      z["ref_s4_pres_in"], relToler=1e-10, absToler=1e-300)
    assert res["status"] == 0 and res["converged"] == 1
    assert rel_l2(pres, z["ref_s5_pres"]) <= PCG_TOL
    assert bitwise(rhs1, z["ref_s5_rhs1"])
    assert bitwise(pdiag, z["ref_s5_pdiag"])
    assert abs(res["iterations"] - int(z["ref_s5_cg"][0])) <= 2


def test_context_solve_pressure():
    """cbs3d_solve_pressure: the drop-in on a context, same inputs and
    side effects as the standalone solver."""
    case, z = load_case(fixture_path("cav6j"))
    c = _gpu().Context(case)
    pres, rhs1, pdiag, res = c.solve_pressure(z["ref_s4_gstif"], z["ref_s4_pdiag_in"], z["ref_s4_rhs1"],
                                              z["ref_s4_pres_in"])
    assert res["status"] == 0 and res["converged"] == 1
    assert rel_l2(pres, z["ref_s5_pres"]) <= PCG_TOL
    assert bitwise(rhs1, z["ref_s5_rhs1"])
    assert bitwise(pdiag, z["ref_s5_pdiag"])
    assert abs(res["iterations"] - int(z["ref_s5_cg"][0])) <= 2
    assert abs(res["initial_l2"] - z["ref_s5_cg"][1]) <= 1e-12 * abs(z["ref_s5_cg"][1])


def test_deterministic_reruns():
    a, _, _ = _ctx("cav6j")
    b, _, _ = _ctx("cav6j")
    a.step(5)
    b.step(5)
    for x, y in zip(a.fields(), b.fields()):
        assert bitwise(x, y)


def test_graph_and_eager_identical():
    a, _, _ = _ctx("chan_sym", use_graph=True)
    b, _, _ = _ctx("chan_sym", use_graph=False)
    a.step(4)
    b.step(4)
    for x, y in zip(a.fields(), b.fields()):
        assert bitwise(x, y)


def test_case_files_contract(tmp_path):
    """The engine's .plt/.bco/.par reader (cbs3d_create_from_case) against
    the in-memory path on the same case."""
    case, z = load_case(fixture_path("cht"))
    base = case.write(str(tmp_path), "cht")
    gpu = _gpu()
    a = gpu.Context(case_name=base)
    b = gpu.Context(case)
    for k in ("detJ", "iside", "color_elem", "bc_list", "wall_node_list"):
        assert bitwise(a.get(k), b.get(k)), k
    a.step(3)
    u, p, t = a.fields()
    assert rel_l2(u, z["ref_final_unkno"]) <= RUN_TOL
    assert rel_l2(t, z["ref_final_temperature"]) <= RUN_TOL


@pytest.mark.parametrize("name", ["cav6j", "cht"])
def test_pcg_variants_bitwise_identical(name):
    """The three PCG kernels (vectors in global memory, register-resident
    rows, shared-memory halo) run the same arithmetic in the same order: at
    the same grid size their results are bit-identical."""
    runs = []
    for k in (1, 2, 3):
        c, _, z = _ctx(name, pcg_kernel=k, pcg_blocks=8)
        c.step(int(z["nsteps"][0]))
        runs.append(c.fields())
    for other in runs[1:]:
        for x, y in zip(runs[0], other):
            assert bitwise(x, y)


MIXED_TOL = 1e-8     # FP32 inner PCG with FP64 defect correction, vs FP64


@pytest.mark.parametrize("name", ["cav6j", "chan_sym", "cht"])
def test_mixed_precision_vs_reference(name):
    """Mixed mode (extension, no reference counterpart): every solve stops
    on the FP64 true residual meeting relToler, so short runs agree with the
    reference's FP64 golden vectors to MIXED_TOL."""
    gpu = _gpu()
    c, _, z = _ctx(name, precision=gpu.MIXED)
    st = c.step(int(z["nsteps"][0]))
    u, p, t = c.fields()
    assert st.cg.outer_sweeps >= 1
    assert rel_l2(u, z["ref_final_unkno"]) <= MIXED_TOL
    assert rel_l2(p, z["ref_final_pres"]) <= MIXED_TOL
    if _param(z, "temp_calc") or _param(z, "material_enabled"):
        assert rel_l2(t, z["ref_final_temperature"]) <= MIXED_TOL


def test_mixed_precision_vs_fp64_jittered_cavity():
    """The benchmark's case family (jittered cavity, Re=400) at 24^3: mixed
    and FP64 engines agree to MIXED_TOL on u and p after 8 steps."""
    from cbs3d import cases
    gpu = _gpu()
    case = cases.cavity(24, re=400.0, ntime=10 ** 6, jitter=0.15, seed=1234)
    a = gpu.Context(case)
    a.step(8)
    b = gpu.Context(case, precision=gpu.MIXED)
    b.step(8)
    (ua, pa, _), (ub, pb, _) = a.fields(), b.fields()
    assert rel_l2(ub, ua) <= MIXED_TOL
    assert rel_l2(pb, pa) <= MIXED_TOL


def test_two_level_matches_jacobi():
    """Two-level preconditioner (extension: Jacobi plus a coarse correction
    on one aggregate per CTA): same stopping test, far fewer iterations, and
    the fields agree with the Jacobi engine to RUN_TOL after 6 steps of the
    48^3 jittered cavity (a mesh large enough for the one-CTA-per-SM kernel)."""
    from cbs3d import cases
    gpu = _gpu()
    case = cases.cavity(48, re=400.0, ntime=10 ** 6, jitter=0.15, seed=1234)
    a = gpu.Context(case)
    sa = a.step(6)
    b = gpu.Context(case, two_level=True)
    sb = b.step(6)
    assert sb.pcg_kernel == 6
    assert sb.cg.iterations < 0.6 * sa.cg.iterations
    assert sb.cg.final_relative_l2 <= case.params["relToler"]
    (ua, pa, _), (ub, pb, _) = a.fields(), b.fields()
    assert rel_l2(ub, ua) <= RUN_TOL
    assert rel_l2(pb, pa) <= RUN_TOL


@pytest.mark.parametrize("g", [1, 37, 148, 160])
def test_coarse_inverse_kernels(g):
    """The two device Gauss-Jordan kernels for the two-level preconditioner's
    aggregated operator (register tiles, the one solves use; shared memory)
    give the same bits, match numpy's inverse of a seeded SPD matrix to 1e-12,
    and treat an empty aggregate (zero row, column and diagonal) as identity."""
    gpu = _gpu()
    rng = np.random.default_rng(7 + g)
    b = rng.standard_normal((g, g))
    a = b @ b.T / g + np.diag(rng.uniform(0.5, 2.0, g))
    if g > 2:
        a[g // 2, :] = 0.0
        a[:, g // 2] = 0.0
    r = gpu.coarse_inverse(a, variant=0)
    s = gpu.coarse_inverse(a, variant=1)
    assert bitwise(r, s)
    a1 = a.copy()
    if g > 2:
        a1[g // 2, g // 2] = 1.0
    ref = np.linalg.inv(a1)
    assert np.linalg.norm(r - ref) / np.linalg.norm(ref) <= 1e-12


@pytest.mark.parametrize("choice,kernel", [(1, 1), (5, 8)])
def test_global_kernel_halo_in_parts(choice, kernel):
    """The global-vector PCG kernels (two grid reductions per iteration, and
    the single-reduction form) with their neighbour values staged in shared
    memory, in several parts per CTA when a CTA's whole halo does not fit
    (forced here: the global kernel on 8 CTAs for a 48^3 cavity, ~14,700 rows
    per CTA): same solutions as the default engine to RUN_TOL, iteration
    counts within 2."""
    from cbs3d import cases
    gpu = _gpu()
    case = cases.cavity(48, re=400.0, ntime=10 ** 6, jitter=0.15, seed=1234)
    a = gpu.Context(case)
    b = gpu.Context(case, pcg_kernel=choice, pcg_blocks=8)
    for _ in range(3):
        sa, sb = a.step(1), b.step(1)
        assert sb.pcg_kernel == kernel
        assert abs(sa.cg.iterations - sb.cg.iterations) <= 2
    (ua, pa, _), (ub, pb, _) = a.fields(), b.fields()
    assert rel_l2(ub, ua) <= RUN_TOL
    assert rel_l2(pb, pa) <= RUN_TOL


@pytest.mark.parametrize("n", [48, 64, 70, 72])
def test_tensor_memory_coefficients_bitwise(n):
    """The register-resident single-reduction PCG reads its rows'
    coefficients from the SM's tensor memory (every row where they all fit,
    else the rows after a shared-memory one) or streams them from L2
    (pcg_kernel=10): the same values enter the same products in the same
    order, so fields and iteration counts agree bit for bit.  48^3 runs two
    rows per thread, 64^3 (the bench mesh) four, 70^3 eight (the first in
    shared memory, the next four in tensor memory, the rest from L2), 72^3
    eight without the shared-memory copy (the first four in tensor memory)."""
    from cbs3d import cases
    gpu = _gpu()
    case = cases.cavity(n, re=400.0, ntime=10 ** 6, jitter=0.15, seed=1234)
    ctxs = [gpu.Context(case, pcg_kernel=k) for k in (10, 11, 0)]
    for _ in range(3):
        st = [c.step(1) for c in ctxs]
        assert [s.pcg_kernel for s in st] == [4, 9, 9]
        assert len({s.cg.iterations for s in st}) == 1
    ref = ctxs[0].fields()
    for c in ctxs[1:]:
        for x, y in zip(ref, c.fields()):
            assert bitwise(x, y)


def test_global_single_reduction_bitwise_equals_register_kernel():
    """The single-reduction PCG with vectors in global memory (the kernel of
    meshes beyond the register tiling) performs, row by row and at the same
    grid, the same operations in the same order as the register-resident
    single-reduction kernel that runs the 64^3 bench: on a 48^3 cavity, where
    both run on the default grid, pressure and velocity agree bit for bit
    after five steps."""
    from cbs3d import cases
    gpu = _gpu()
    case = cases.cavity(48, re=400.0, ntime=10 ** 6, jitter=0.15, seed=1234)
    a = gpu.Context(case, pcg_kernel=4)
    b = gpu.Context(case, pcg_kernel=5)
    for _ in range(5):
        sa, sb = a.step(1), b.step(1)
        assert sa.pcg_kernel in (4, 9) and sb.pcg_kernel == 8
        assert sa.cg.iterations == sb.cg.iterations
    for x, y in zip(a.fields(), b.fields()):
        assert bitwise(x, y)


def test_large_mesh_runs_single_reduction_global_kernel():
    """Beyond the register tiling (88^3 cavity: 704,969 nodes on 148 SMs) the
    engine runs the single-reduction global-vector kernel by itself; after
    two steps it agrees with the two-reduction kernel to RUN_TOL, with
    iteration counts within 2."""
    from cbs3d import cases
    gpu = _gpu()
    case = cases.cavity(88, re=400.0, ntime=10 ** 6, jitter=0.15, seed=1234)
    a = gpu.Context(case)
    b = gpu.Context(case, pcg_kernel=1)
    for _ in range(2):
        sa, sb = a.step(1), b.step(1)
        assert sa.pcg_kernel == 8 and sb.pcg_kernel == 1
        assert abs(sa.cg.iterations - sb.cg.iterations) <= 2
    (ua, pa, _), (ub, pb, _) = a.fields(), b.fields()
    assert rel_l2(ua, ub) <= RUN_TOL
    assert rel_l2(pa, pb) <= RUN_TOL
