"""Aggregation-multigrid preconditioned CG (extension; the reference's
counterpart is its PETSc/AMG pressure path, solver_opt=3): a V(1,1) cycle on
aggregates of 8 Morton-ordered rows with Galerkin coarse operators, under
the reference's CG stopping test.  It must reach the same solutions as the
Jacobi engine, need few iterations, and give the same bits and iteration
counts for any grid size."""
import numpy as np
import pytest

from helpers import fixture_path, load_case, rel_l2

pytestmark = pytest.mark.gpu

RUN_TOL = 1e-8


def _gpu():
    from cbs3d import gpu
    return gpu


def test_multigrid_cavity64_200_steps_vs_jacobi():
    """The benchmark cavity (64^3 hexes x 6 tets, jitter 0.15h, Re 400):
    at most 80 iterations per step, and u, p within RUN_TOL of the Jacobi
    engine after 200 steps."""
    from cbs3d import cases
    gpu = _gpu()
    case = cases.cavity(64, re=400.0, ntime=10 ** 6, jitter=0.15, seed=1234)
    a = gpu.Context(case)
    a.step(200)
    b = gpu.Context(case, multigrid=True)
    its = []
    for _ in range(200):
        st = b.step(1)
        its.append(st.cg.iterations)
        assert st.cg.final_relative_l2 <= case.params["relToler"]
    assert st.pcg_kernel == 7
    print("multigrid iterations per step: max", max(its), "mean", np.mean(its))
    assert max(its) <= 80
    (ua, pa, _), (ub, pb, _) = a.fields(), b.fields()
    assert rel_l2(ub, ua) <= RUN_TOL
    assert rel_l2(pb, pa) <= RUN_TOL


@pytest.mark.parametrize("blocks", [97, 50])
def test_multigrid_independent_of_grid_size(blocks):
    """The hierarchy and every reduction order depend on the mesh only: a
    32^3 jittered cavity gives bitwise equal fields and equal iteration
    counts on the full grid and on a smaller one."""
    from cbs3d import cases
    gpu = _gpu()
    case = cases.cavity(32, re=400.0, ntime=10 ** 6, jitter=0.15, seed=1234)
    a = gpu.Context(case, multigrid=True)
    b = gpu.Context(case, multigrid=True, pcg_blocks=blocks)
    for _ in range(5):
        sa, sb = a.step(1), b.step(1)
        assert sa.pcg_kernel == sb.pcg_kernel == 7
        assert sa.cg.iterations == sb.cg.iterations
    (ua, pa, _), (ub, pb, _) = a.fields(), b.fields()
    assert np.array_equal(ua, ub)
    assert np.array_equal(pa, pb)


def test_multigrid_cavity16_500_steps_vs_reference():
    """The 16^3 cavity (500 steps, Re 100): the reference's fields to
    RUN_TOL with a fraction of its iterations."""
    gpu = _gpu()
    case, z = load_case(fixture_path("c1_cavity16"))
    ctx = gpu.Context(case, multigrid=True)
    st = ctx.step(500)
    assert st.pcg_kernel == 7
    u, p, _ = ctx.fields()
    assert rel_l2(u, z["ref_final_unkno"]) <= RUN_TOL
    assert rel_l2(p, z["ref_final_pres"]) <= RUN_TOL
    hist = z["ref_history"].reshape(-1, 21)
    assert st.cg_iterations_total < 0.4 * hist[:, 1].sum()


def test_multigrid_pressure_solver_drop_in():
    """cbs3d_pcg_solve with the multigrid option on a pressure system of the
    24^3 jittered cavity: the Jacobi drop-in's solution to PCG tolerance in
    under half its iterations.  The drop-in has no coordinates, so its rows
    follow a breadth-first order and its aggregates are less compact than
    the Morton-ordered ones of a context (measured: 115 against 281)."""
    from cbs3d import cases
    gpu = _gpu()
    case = cases.cavity(24, re=400.0, ntime=10 ** 6, jitter=0.15, seed=1234)
    ctx = gpu.Context(case)
    ctx.step(3)
    for st in ("begin_step", "time_step", "lhs", "step1", "step2_rhs"):
        ctx.stage(st)
    gstif, pdiag, rhs1, pres = ctx.get("gstif"), ctx.get("pdiag"), ctx.get("rhs1"), ctx.get("pres")
    m = case.mesh
    bl, bv = ctx.get("bc_list"), ctx.get("bc_values")
    ja = gpu.PressureSolver(m.intma, m.mat_elem, bl, bv)
    jm = gpu.PressureSolver(m.intma, m.mat_elem, bl, bv, multigrid=True)
    pa, _, _, ra = ja.solve(gstif, pdiag, rhs1, pres)
    pm, _, _, rm = jm.solve(gstif, pdiag, rhs1, pres)
    assert ra["converged"] and rm["converged"]
    assert rm["iterations"] < 0.5 * ra["iterations"]
    assert rel_l2(pm, pa) <= RUN_TOL


def test_multigrid_falls_back_on_tiny_mesh():
    """A mesh whose rows fit the dense coarsest level alone (4^3 cavity,
    125 nodes) has no hierarchy: the option leaves the Jacobi engine."""
    gpu = _gpu()
    case, _ = load_case(fixture_path("cav4"))
    a = gpu.Context(case)
    b = gpu.Context(case, multigrid=True)
    sa, sb = a.step(3), b.step(3)
    assert sb.pcg_kernel != 7
    assert sa.cg.iterations == sb.cg.iterations
