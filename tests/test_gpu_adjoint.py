"""Body force, tangent-linear and adjoint runs (extension, no reference
counterpart).  The forward body-force path is pinned against the oracle
(which carries the same extension); derivatives are pinned by central
finite differences, by the tangent-linear pass (adjoint . dir == TLM), and by
checkpoint-interval invariance of the adjoint.  A torch.autograd.Function
over the C ABI -- test harness only -- checks that the adjoint drops into
autograd."""
import numpy as np
import pytest

from helpers import bitwise, rel_l2

pytestmark = pytest.mark.gpu

FD_TOL = 1e-6        # adjoint/TLM against central finite differences
TLM_TOL = 1e-9       # adjoint . direction against the TLM directional derivative
FWD_TOL = 1e-8       # body-force forward against the oracle (PCG tolerance)


def _small():
    from cbs3d import cases
    c = cases.channel_adjoint(12, 4, 4, length=3.0, re=100.0, dtfix=0.02, ntime=100, rel_tol=1e-13)
    return c, cases.region_weights(c, lo=1.5, hi=2.5), cases.body_force(c, seed=11)


def _ctx(case, f):
    from cbs3d import gpu
    ctx = gpu.Context(case)
    ctx.set_body_force(f)
    return ctx


def test_body_force_forward_vs_oracle():
    from oracle import pyoracle
    case, _, f = _small()
    ctx = _ctx(case, f)
    ctx.step(5)
    u, p, _ = ctx.fields()
    orc = pyoracle.Oracle(case)
    orc.set("bforce", f)
    orc.step(5)
    assert rel_l2(u, orc.get("unkno")) <= FWD_TOL
    assert rel_l2(p, orc.get("pres")) <= FWD_TOL
    # a zero body force is the plain step, bit for bit
    from cbs3d import gpu
    a = gpu.Context(case)
    a.step(3)
    b = _ctx(case, np.zeros_like(f))
    b.step(3)
    for x, y in zip(a.fields(), b.fields()):
        assert bitwise(x, y)


def _fd(ctx, f, d, nsteps, w, h):
    ctx.set_body_force(f + h * d)
    jp = ctx.objective(nsteps, w)
    ctx.set_body_force(f - h * d)
    jm = ctx.objective(nsteps, w)
    ctx.set_body_force(f)
    return (jp - jm) / (2.0 * h)


def test_tlm_and_adjoint_vs_finite_differences():
    case, w, f = _small()
    ctx = _ctx(case, f)
    n = 8
    J0, grad = ctx.adjoint(n, w, every=3)
    assert J0 == ctx.objective(n, w)
    rng = np.random.default_rng(5)
    for _ in range(4):
        d = rng.normal(0.0, 1.0, size=f.size)
        fd = _fd(ctx, f, d, n, w, 1e-6)
        J, dj = ctx.tlm(n, w, d)
        assert J == J0
        ad = float(grad @ d)
        assert abs(dj - fd) <= FD_TOL * abs(fd)
        assert abs(ad - fd) <= FD_TOL * abs(fd)
        assert abs(ad - dj) <= TLM_TOL * abs(dj)


def test_adjoint_invariant_to_checkpoint_interval():
    case, w, f = _small()
    ctx = _ctx(case, f)
    ref = ctx.adjoint(7, w, every=1)
    for every in (2, 3, 7, 50):
        J, g = ctx.adjoint(7, w, every=every)
        assert J == ref[0] and bitwise(g, ref[1])
    # the runs leave the state where it was
    u0 = ctx.fields()
    ctx.tlm(3, w, f)
    for x, y in zip(u0, ctx.fields()):
        assert bitwise(x, y)


def test_adjoint_needs_fixed_time_step():
    from cbs3d import cases, gpu
    c = cases.channel(8, 4, 4, length=2.0, ntime=10)
    ctx = gpu.Context(c)
    with pytest.raises(gpu.CBSError):
        ctx.adjoint(2, np.ones(c.mesh.npoin))


def test_autograd_wrapper():
    """dJ/df through torch.autograd (harness-only Function over the C ABI)."""
    import torch
    case, w, f = _small()
    ctx = _ctx(case, f)
    n = 6

    class CBSObjective(torch.autograd.Function):
        @staticmethod
        def forward(fctx, force):
            ctx.set_body_force(force.detach().numpy())
            J, g = ctx.adjoint(n, w, every=2)
            fctx.save_for_backward(torch.from_numpy(g))
            return torch.tensor(J, dtype=torch.float64)

        @staticmethod
        def backward(fctx, gJ):
            (g,) = fctx.saved_tensors
            return gJ * g

    x = torch.tensor(f, dtype=torch.float64, requires_grad=True)
    J = CBSObjective.apply(x)
    J.backward()
    d = np.random.default_rng(9).normal(0.0, 1.0, size=f.size)
    fd = _fd(ctx, f, d, n, w, 1e-6)
    assert abs(float(x.grad.numpy() @ d) - fd) <= FD_TOL * abs(fd)


def test_channel_config_adjoint_200_steps():
    """The adjoint-sensitivity channel at full size: [0,6]x[0,1]^2, 96x16x16
    hexes x 6 tets (147,456 tets, 28,033 nodes), nu = 0.01, seeded body force
    N(0, 0.01^2), J = mean kinetic energy over 4 <= x <= 5 after 200 fixed-dt
    steps; adjoint with a checkpoint every 20 steps against the tangent-linear
    pass and central finite differences along 16 seeded standard-normal
    directions, every direction held to every gate:
      * adjoint . d against the tangent-linear derivative: 1e-9;
      * central differences at h = 1e-4: 1e-7;
      * central differences at h = 1e-6: 1e-6.
    J is summed over the nodes with compensated summation: with a plain
    running sum its rounding (several ulp of J, different for J(f + h d) and
    J(f - h d)) put one direction at 1.6e-6 at h = 1e-6; compensated, the
    worst direction measures 9e-8."""
    from cbs3d import cases
    case = cases.channel_adjoint()
    w = cases.region_weights(case)
    f = cases.body_force(case)
    ctx = _ctx(case, f)
    n = 200
    J0, grad = ctx.adjoint(n, w, every=20)
    rng = np.random.default_rng(2024)
    errs6, errs4, errst = [], [], []
    for _ in range(16):
        d = rng.normal(0.0, 1.0, size=f.size)
        ad = float(grad @ d)
        errs6.append(abs(ad - _fd(ctx, f, d, n, w, 1e-6)) / abs(ad))
        errs4.append(abs(ad - _fd(ctx, f, d, n, w, 1e-4)) / abs(ad))
        _, dj = ctx.tlm(n, w, d)
        errst.append(abs(ad - dj) / abs(dj))
    print("FD h=1e-6:", " ".join(f"{e:.1e}" for e in errs6))
    print("FD h=1e-4:", " ".join(f"{e:.1e}" for e in errs4))
    print("TLM:      ", " ".join(f"{e:.1e}" for e in errst))
    assert max(errst) <= TLM_TOL, errst
    assert max(errs4) <= 0.1 * FD_TOL, errs4
    assert max(errs6) <= FD_TOL, errs6


# ------------------------------------------------- heat-flux sensitivities
def _cht_small():
    from cbs3d import cases
    c = cases.cht_slab(8, 4, 2, 2, length=2.0, ntime=100)
    w = cases.region_weights(c, axis=0, lo=2.0, hi=2.0)
    w[c.mesh.coord.reshape(-1, 3)[:, 1] < 0.0] = 0.0
    w /= w.sum()
    return c, w


def test_uniform_face_heat_flux_is_the_plain_step():
    from cbs3d import gpu
    case, _ = _cht_small()
    a = gpu.Context(case)
    a.step(4)
    b = gpu.Context(case)
    b.set_face_heat_flux(np.full(b.heat_flux_faces(), case.params["heat_flux_bc"]))
    b.step(4)
    for x, y in zip(a.fields(), b.fields()):
        assert bitwise(x, y)


def test_heat_adjoint_vs_tlm_and_finite_differences():
    from cbs3d import gpu
    case, w = _cht_small()
    ctx = gpu.Context(case)
    nf = ctx.heat_flux_faces()
    q = 1.0 + 0.1 * np.random.default_rng(3).uniform(-1.0, 1.0, nf)
    ctx.set_face_heat_flux(q)
    n = 9
    J0, g = ctx.heat_adjoint(n, w, every=4)
    assert J0 == ctx.heat_objective(n, w)
    J1, g1 = ctx.heat_adjoint(n, w, every=1)
    assert J1 == J0 and bitwise(g, g1)
    rng = np.random.default_rng(8)
    for _ in range(3):
        d = rng.normal(0.0, 1.0, nf)
        _, dj = ctx.heat_tlm(n, w, d)
        ad = float(g @ d)
        assert abs(ad - dj) <= TLM_TOL * abs(dj)
        h = 1e-2   # J is affine in q: exact differences at any step
        ctx.set_face_heat_flux(q + h * d)
        jp = ctx.heat_objective(n, w)
        ctx.set_face_heat_flux(q - h * d)
        jm = ctx.heat_objective(n, w)
        ctx.set_face_heat_flux(q)
        fd = (jp - jm) / (2 * h)
        assert abs(ad - fd) <= 1e-8 * abs(fd)


def test_cht_config_heat_flux_gradient():
    """Conjugate heat transfer at full size: fluid [0,4]x[0,1]x[0,1] over a
    solid slab, 128x(24+6)x24 hexes x 6 tets (552,960 tets), parabolic inlet
    with T=0, outlet p=0, uniform flux on y=-0.25 perturbed per face by a
    seeded +-10%, k_s/k_f=10, Pr=0.71, Re=200, 300 steps.  J = mean outlet
    temperature (fluid nodes on x=4); its gradient with respect to every face
    flux from the adjoint (checkpoint every 30 steps) against the
    tangent-linear pass and central differences along 4 seeded directions.
    The temperature does not act on the flow, so J is affine in the fluxes
    and central differences are exact up to rounding at any step: h = 1e-2
    keeps the forward rounding noise (about 1e-12 in J after 300 steps) out
    of the comparison, which is then held to 1e-8.  The mixed-precision
    engine's outlet temperature after the same steps agrees with FP64 to
    1e-8."""
    from cbs3d import cases, gpu
    case = cases.cht_slab(128, 24, 6, 24, length=4.0, re=200.0, pr=0.71, k_ratio=10.0, q=1.0, ntime=300)
    xy = case.mesh.coord.reshape(-1, 3)
    w = ((np.abs(xy[:, 0] - 4.0) < 1e-12) & (xy[:, 1] >= 0.0)).astype(float)
    w /= w.sum()
    ctx = gpu.Context(case)
    nf = ctx.heat_flux_faces()
    assert nf == 2 * 128 * 24
    q = 1.0 + 0.1 * np.random.default_rng(55).uniform(-1.0, 1.0, nf)
    ctx.set_face_heat_flux(q)
    n = 300
    J0, g = ctx.heat_adjoint(n, w, every=30)
    rng = np.random.default_rng(77)
    for k in range(4):
        d = rng.normal(0.0, 1.0, nf)
        ad = float(g @ d)
        if k == 0:
            _, dj = ctx.heat_tlm(n, w, d)
            assert abs(ad - dj) <= TLM_TOL * abs(dj)
        ctx.set_face_heat_flux(q + 1e-2 * d)
        jp = ctx.heat_objective(n, w)
        ctx.set_face_heat_flux(q - 1e-2 * d)
        jm = ctx.heat_objective(n, w)
        ctx.set_face_heat_flux(q)
        fd = (jp - jm) / 2e-2
        assert abs(ad - fd) <= 1e-8 * abs(fd), (k, ad, fd)
    m = gpu.Context(case, precision=gpu.MIXED)
    m.set_face_heat_flux(q)
    assert abs(m.heat_objective(n, w) - J0) <= 1e-8 * abs(J0)
