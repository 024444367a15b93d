"""Seeded synthetic CBS3D cases on Kuhn-tetrahedral box meshes.

A box is split into nx*ny*nz hexahedra, each cut into the six Kuhn
tetrahedra that share the hex diagonal (0,0,0)->(1,1,1).  Connectivity is
made positively oriented by swapping local nodes 2 and 3 where needed, the
rule the reference exporter applies (tools/export_cbs3d_tet.py:225-249).
Boundary triangles carry raw side ids that a .bco file maps to solver BC ids
(src/io/MeshIO.cpp:872-982); the default cube ids are 1 xmin, 2 xmax,
3 ymin, 4 ymax (lid), 5 zmin, 6 zmax (tools/export_cbs3d_tet.py:24-30).

The writers emit the positional grammar MeshIO reads:
  .plt  NELEM NPOIN NBOUN / eid n1..n4 / nid x y z / f1 f2 f3 parent raw_id
        (src/io/MeshIO.cpp:713-868)
  .bco  NFLAG MASS_CHECK / raw_id solver_bc           (src/io/MeshIO.cpp:872-982)
  .par  label/value pairs in fixed order               (src/io/MeshIO.cpp:986-1437)
  .material / .matprop for conjugate heat transfer     (src/io/MeshIO.cpp:1441-1623)
"""

from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

# The six axis orders of a Kuhn split: tet = (v0, v0+e_a, v0+e_a+e_b, v7).
_KUHN_PERMS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))
_EVEN = {(0, 1, 2), (1, 2, 0), (2, 0, 1)}

# Local face f (0-based) is opposite local node f; node order as the exporter
# writes it so that a positively oriented tet yields outward triangles.
_FACE_NODES = ((1, 2, 3), (0, 3, 2), (0, 1, 3), (0, 2, 1))


@dataclass
class Mesh:
    coord: np.ndarray          # (N,3) float64
    intma: np.ndarray          # (E,4) int32, 1-based node ids
    bfaces: np.ndarray         # (NB,5) int32: n1 n2 n3 parent(1-based) raw_side_id
    lattice: np.ndarray        # (N,3) int64 lattice coordinates
    shape: tuple               # (nx, ny, nz)
    mat_elem: np.ndarray = None  # (E,) int32 material ids (0 fluid)

    @property
    def nelem(self) -> int:
        return int(self.intma.shape[0])

    @property
    def npoin(self) -> int:
        return int(self.coord.shape[0])

    @property
    def nboun(self) -> int:
        return int(self.bfaces.shape[0])


def default_side_id(plane: int, centroid: np.ndarray) -> np.ndarray:
    """Cube-face ids 1..6 for planes xmin,xmax,ymin,ymax,zmin,zmax."""
    return np.full(centroid.shape[0], plane + 1, dtype=np.int32)


def box_mesh(nx: int, ny: int, nz: int, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0),
             jitter: float = 0.0, seed: int = 1234, side_id=default_side_id,
             axis_coords=None) -> Mesh:
    """Kuhn mesh of the box [lo,hi]; interior nodes jittered by U(-jitter*h, jitter*h).
    axis_coords=(xs, ys, zs) optionally gives explicit grid lines per axis."""
    nx, ny, nz = int(nx), int(ny), int(nz)
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    npx, npy, npz = nx + 1, ny + 1, nz + 1
    k, j, i = np.meshgrid(np.arange(npz), np.arange(npy), np.arange(npx), indexing="ij")
    lat = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.int64)
    h = (hi - lo) / np.array([nx, ny, nz], dtype=np.float64)
    coord = lo[None, :] + lat.astype(np.float64) * h[None, :]
    # exact end planes (no rounding drift on the hi faces)
    for d, n in enumerate((nx, ny, nz)):
        coord[lat[:, d] == n, d] = hi[d]
    if axis_coords is not None:
        for d in range(3):
            if axis_coords[d] is not None:
                coord[:, d] = np.asarray(axis_coords[d], dtype=np.float64)[lat[:, d]]
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        disp = rng.uniform(-jitter, jitter, size=coord.shape) * h[None, :]
        interior = ((lat[:, 0] > 0) & (lat[:, 0] < nx) & (lat[:, 1] > 0) & (lat[:, 1] < ny)
                    & (lat[:, 2] > 0) & (lat[:, 2] < nz))
        coord[interior] += disp[interior]

    def nid(ii, jj, kk):
        return 1 + ii + npx * (jj + npy * kk)

    hk, hj, hi_ = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    hi_, hj, hk = hi_.ravel(), hj.ravel(), hk.ravel()
    nhex = hi_.size
    intma = np.empty((nhex, 6, 4), dtype=np.int64)
    for p, perm in enumerate(_KUHN_PERMS):
        v = [np.stack([hi_, hj, hk], axis=1)]
        cur = v[0].copy()
        for a in perm:
            cur = cur.copy()
            cur[:, a] += 1
            v.append(cur)
        ids = [nid(w[:, 0], w[:, 1], w[:, 2]) for w in (v[0], v[1], v[2], v[3])]
        if perm not in _EVEN:
            ids = [ids[0], ids[2], ids[1], ids[3]]
        intma[:, p, :] = np.stack(ids, axis=1)
    intma = intma.reshape(-1, 4)

    # orientation check after jitter (swap 2<->3 where a jittered tet flipped)
    x = coord[intma - 1]
    d1, d2, d3 = x[:, 1] - x[:, 0], x[:, 2] - x[:, 0], x[:, 3] - x[:, 0]
    vol6 = np.einsum("ij,ij->i", d1, np.cross(d2, d3))
    if np.any(np.abs(vol6) < 1e-14):
        raise ValueError("degenerate tetrahedron in generated mesh")
    neg = vol6 < 0
    if np.any(neg):
        intma[neg] = intma[neg][:, [0, 2, 1, 3]]

    # boundary triangles: tet faces whose three nodes share a boundary plane
    nelem = intma.shape[0]
    latn = lat[intma - 1]  # (E,4,3)
    faces = []
    bounds = ((0, 0), (0, nx), (1, 0), (1, ny), (2, 0), (2, nz))
    for f, fn in enumerate(_FACE_NODES):
        fl = latn[:, list(fn), :]  # (E,3,3)
        for plane, (d, val) in enumerate(bounds):
            on = np.all(fl[:, :, d] == val, axis=1)
            if not np.any(on):
                continue
            e = np.nonzero(on)[0]
            nodes = intma[e][:, list(fn)]
            cen = coord[nodes - 1].mean(axis=1)
            sid = side_id(plane, cen)
            faces.append(np.column_stack([e, np.full(e.size, f), nodes, e + 1, sid]))
    bf = np.concatenate(faces, axis=0)
    order = np.lexsort((bf[:, 1], bf[:, 0]))  # element order, then local face
    bf = bf[order][:, 2:].astype(np.int32)
    return Mesh(coord=coord, intma=intma.astype(np.int32), bfaces=bf, lattice=lat,
                shape=(nx, ny, nz), mat_elem=np.zeros(nelem, dtype=np.int32))


# ---------------------------------------------------------------------------
# .par parameters (field order of src/io/MeshIO.cpp:986-1191)
# ---------------------------------------------------------------------------

def default_params(**over) -> dict:
    p = dict(
        solver_opt=1, restart_opt=0, temp_calc=0,
        cinf=(0.0, 0.0, 0.0, 0.0, 0.0),
        ntime=10, transient_on=0, dtfixed=0, dtfix=1.0, iwrite=1,
        csafm=0.5, theta1=1.0,
        cbs_scheme=1, ilots=1, htype=1, step2_check=0, rem_deltp=0, beta_opt=1,
        dtfix_end=0, csafm2=2.0, epsilon1=1.0e-6, deltr=1.0e20,
        re=100.0, pr=0.71, ra=0.0, ri=0.0,
        convection_type=0, pnode=1,
        write_output=0, write_time_output=0.0, time_output_interval=0.0, end_rtime=0.0,
        relToler=1.0e-10, absToler=1.0e-300,
        vel_check=0, l2v=0.0, temp_check=0, l2T=0.0,
        paraview=0, tecplot=0, nusselt_calc=0, nusselt_flag=0,
        runtime_mod=0,
        alpha_sf=1.0, k_ratio=1.0, source_solid=1.0, heat_flux_bc=0.0,
        dimensional_mode=0, material_enabled=0, massflow_enabled=0,
        p_ref=0.0, model_depth=1.0, mdot=0.0, rho_in=1.0, T_in=0.0, p_out=0.0,
        inlet_u=1.0, inlet_v=0.0, inlet_w=0.0,
        Tinf=25.0, Tref=100.0, Dnu=1.0,
        cg_precond=1, cg_conv_test=2, cg_max_iter=100000, l2p=0.0,
        reslog=1, reslog_every=1, console_every=0, live_plot=0,
        vtu=0, vtu_every=0, vtu_time=0.0, dbg_arrays=0, steady_min=None,
        art_diff=0,
    )
    p.update(over)
    if p["steady_min"] is None:
        p["steady_min"] = p["ntime"]
    return p


def _g(v) -> str:
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    return repr(float(v))


def par_text(p: dict) -> str:
    rows = [
        ("SOLVER_OPT", [p["solver_opt"]]),
        ("RESTART_OPT", [p["restart_opt"]]),
        ("TEMP_CALC", [p["temp_calc"]]),
        ("UX UY UZ P T", list(p["cinf"])),
        ("NTIME TRANSIENT_ON DTFIXED DTFIX IWRITE",
         [p["ntime"], p["transient_on"], p["dtfixed"], p["dtfix"], p["iwrite"]]),
        ("CSAFM THETA1", [p["csafm"], p["theta1"]]),
        ("CBS_SCHEME ILOTS HTYPE STEP2_CHECK REM_DELTP BETA_OPT DTFIX_END CSAFM2 EPSILON1 DELTR",
         [p["cbs_scheme"], p["ilots"], p["htype"], p["step2_check"], p["rem_deltp"], p["beta_opt"],
          p["dtfix_end"], p["csafm2"], p["epsilon1"], p["deltr"]]),
        ("RE PR RA RI", [p["re"], p["pr"], p["ra"], p["ri"]]),
        ("CONVECTION_TYPE", [p["convection_type"]]),
        ("PNODE", [p["pnode"]]),
        ("WRITE_OUTPUT WRITE_TIME_OUTPUT TIME_OUTPUT_INTERVAL END_RTIME",
         [p["write_output"], p["write_time_output"], p["time_output_interval"], p["end_rtime"]]),
        ("RELTOLER ABSTOLER", [p["relToler"], p["absToler"]]),
        ("VEL_CHECK L2V TEMP_CHECK L2T", [p["vel_check"], p["l2v"], p["temp_check"], p["l2T"]]),
        ("PARAVIEW TECPLOT NUSSELT_CALC NUSSELT_FLAG",
         [p["paraview"], p["tecplot"], p["nusselt_calc"], p["nusselt_flag"]]),
        ("RUNTIME_MOD", [p["runtime_mod"]]),
        ("ALPHA_SF K_RATIO SOURCE_SOLID HEAT_FLUX_BC",
         [p["alpha_sf"], p["k_ratio"], p["source_solid"], p["heat_flux_bc"]]),
        ("DIMENSIONAL_MODE MATERIAL_PROPERTIES_ENABLED MASS_FLOW_INLET_ENABLED",
         [p["dimensional_mode"], p["material_enabled"], p["massflow_enabled"]]),
        ("P_REF MODEL_DEPTH MDOT RHO_IN T_IN P_OUT",
         [p["p_ref"], p["model_depth"], p["mdot"], p["rho_in"], p["T_in"], p["p_out"]]),
        ("INLET_U INLET_V INLET_W", [p["inlet_u"], p["inlet_v"], p["inlet_w"]]),
        ("NUSSELT_TINF NUSSELT_TREF NUSSELT_D", [p["Tinf"], p["Tref"], p["Dnu"]]),
        ("CG_PRECOND CG_CONV_TEST CG_MAX_ITER L2NORM_PRES_TOL",
         [p["cg_precond"], p["cg_conv_test"], p["cg_max_iter"], p["l2p"]]),
        ("RESLOG EVERY CONSOLE LIVE VTU VTU_IT VTU_T DBG STEADY_MIN",
         [p["reslog"], p["reslog_every"], p["console_every"], p["live_plot"], p["vtu"],
          p["vtu_every"], p["vtu_time"], p["dbg_arrays"], p["steady_min"]]),
        ("ART_DIFF", [p["art_diff"]]),
    ]
    out = []
    for label, vals in rows:
        out.append(label)
        out.append(" ".join(_g(v) for v in vals))
    return "\n".join(out) + "\n"


@dataclass
class Case:
    mesh: Mesh
    bc_map: dict                      # raw side id -> solver BC id
    params: dict
    materials: dict = field(default_factory=dict)  # id -> (name, phase, rho, cp, k, mu, Qvol)

    def write(self, directory: str, name: str) -> str:
        """Write the case files; returns the case base path."""
        os.makedirs(directory, exist_ok=True)
        base = os.path.join(directory, name)
        write_plt(base + ".plt", self.mesh)
        with open(base + ".bco", "w") as f:
            f.write(f"{len(self.bc_map)} 0\n")
            for raw in sorted(self.bc_map):
                f.write(f"{raw} {self.bc_map[raw]}\n")
        with open(base + ".par", "w") as f:
            f.write(par_text(self.params))
        if self.params.get("material_enabled", 0) > 0:
            m = self.mesh
            with open(base + ".material", "w") as f:
                f.write(f"{m.nelem}\n")
                rows = np.column_stack([np.arange(1, m.nelem + 1), m.intma, m.mat_elem])
                f.write("\n".join(" ".join(str(int(v)) for v in r) for r in rows))
                f.write("\n")
            with open(base + ".matprop", "w") as f:
                f.write(f"{len(self.materials)}\n")
                for mid in sorted(self.materials):
                    name_, phase, rho, cp, k, mu, q = self.materials[mid]
                    f.write(f"{mid} {name_} {phase} {_g(rho)} {_g(cp)} {_g(k)} {_g(mu)} {_g(q)}\n")
        return base


def write_plt(path: str, m: Mesh) -> None:
    with open(path, "w") as f:
        f.write(f"{m.nelem} {m.npoin} {m.nboun}\n")
        e = np.column_stack([np.arange(1, m.nelem + 1), m.intma])
        np.savetxt(f, e, fmt="%d")
        ids = np.arange(1, m.npoin + 1)
        # %.17g round-trips every double exactly through operator>>
        lines = [f"{i} {x!r} {y!r} {z!r}" for i, (x, y, z) in zip(ids.tolist(), m.coord.tolist())]
        f.write("\n".join(lines))
        f.write("\n")
        np.savetxt(f, m.bfaces, fmt="%d")


# ---------------------------------------------------------------------------
# Named configurations
# ---------------------------------------------------------------------------

CAVITY_BC = {1: 530, 2: 530, 3: 530, 4: 500, 5: 530, 6: 530}


def cavity(n: int, re: float = 100.0, ntime: int = 10, jitter: float = 0.0,
           seed: int = 1234, **over) -> Case:
    """Lid-driven cavity: lid y=1 moving with u=(1,0,0), five no-slip walls,
    pressure pinned at node (0,0,0) (pnode=1, no BC 520)."""
    m = box_mesh(n, n, n, jitter=jitter, seed=seed)
    p = default_params(re=re, ntime=ntime, pnode=1, inlet_u=1.0, inlet_v=0.0, inlet_w=0.0, **over)
    return Case(mesh=m, bc_map=dict(CAVITY_BC), params=p)


def cavity_batch(count: int = 48, n_lo: int = 10, n_hi: int = 40, re_lo: float = 50.0, re_hi: float = 1000.0,
                 seed: int = 2024, ntime: int = 100, rel_tol: float = 1.0e-8, **over) -> list:
    """Independent lid-driven cavities of uneven size for the batched step:
    hexes per side uniform in {n_lo..n_hi}, Re log-uniform in [re_lo, re_hi]
    (nu = 1/Re, lid speed 1), each pressure solve to rel_tol, all from one
    seed.  Returns the cases; their sizes and Re are in .mesh and .params."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_lo, n_hi + 1, size=count)
    res = np.exp(rng.uniform(np.log(re_lo), np.log(re_hi), size=count))
    return [cavity(int(n), re=float(r), ntime=ntime, relToler=rel_tol, **over) for n, r in zip(ns, res)]


def channel_adjoint(nx: int = 96, ny: int = 16, nz: int = 16, length: float = 6.0, re: float = 100.0,
                    dtfix: float = 0.01, ntime: int = 200, rel_tol: float = 1.0e-13, **over) -> Case:
    """Channel for the body-force sensitivities: parabolic inlet (BC 508,
    u_max 1) at x=0, zero-pressure outlet (520) at x=L, no-slip walls, nu =
    1/Re, and a fixed time step dtfix (the tangent and adjoint runs need one)."""
    return channel(nx, ny, nz, length=length, re=re, ntime=ntime, dtfixed=1, dtfix=dtfix, relToler=rel_tol, **over)


def region_weights(case: Case, axis: int = 0, lo: float = 4.0, hi: float = 5.0) -> np.ndarray:
    """Objective weights of a mean over the nodes with lo <= x_axis <= hi:
    J = 1/2 sum w_i |u_i|^2 is then their mean kinetic energy."""
    x = case.mesh.coord.reshape(-1, 3)[:, axis]
    sel = (x >= lo - 1e-12) & (x <= hi + 1e-12)
    w = np.zeros(case.mesh.npoin)
    w[sel] = 1.0 / max(int(sel.sum()), 1)
    return w


def body_force(case: Case, sigma: float = 0.01, seed: int = 4321) -> np.ndarray:
    """Seeded per-node body force, every component ~ N(0, sigma^2), node-major."""
    return np.random.default_rng(seed).normal(0.0, sigma, size=3 * case.mesh.npoin)


def channel(nx: int = 96, ny: int = 16, nz: int = 16, length: float = 6.0, re: float = 100.0,
            ntime: int = 10, symmetry_z: bool = False, **over) -> Case:
    """Channel [0,L]x[0,1]x[0,1]: BC 508 parabolic inlet at x=0, BC 520 outlet
    at x=L, no-slip (530) elsewhere, optionally symmetry (506) on the z faces."""
    m = box_mesh(nx, ny, nz, hi=(length, 1.0, 1.0))
    bc = {1: 508, 2: 520, 3: 530, 4: 530, 5: 506 if symmetry_z else 530,
          6: 506 if symmetry_z else 530}
    p = default_params(re=re, ntime=ntime, **over)
    return Case(mesh=m, bc_map=bc, params=p)


def cht_slab(nx: int = 128, ny_fluid: int = 24, ny_solid: int = 6, nz: int = 24,
             length: float = 4.0, re: float = 200.0, pr: float = 0.71, k_ratio: float = 10.0,
             q: float = 1.0, ntime: int = 10, **over) -> Case:
    """Conjugate heat transfer: fluid box [0,L]x[0,1]x[0,1] on a solid slab
    [0,L]x[-0.25,0]x[0,1].  Fluid inlet BC 508 (u=6y(1-y), T=0) at x=0, fluid
    outlet BC 520 at x=L, heat flux BC 532 (q) on y=-0.25, walls 530 elsewhere.
    Dimensional material mode: fluid rho=cp=1, mu=1/Re, k=1/(Re Pr); solid
    rho=cp=1, mu=0, k=k_ratio*k_fluid."""
    ny = ny_fluid + ny_solid
    y0 = -0.25
    ys = np.concatenate([y0 - y0 * np.arange(ny_solid) / ny_solid,
                         np.arange(ny_fluid + 1) / ny_fluid])
    # raw ids: 1 fluid inlet, 2 fluid outlet, 3 heated bottom, 4 top, 5/6 z walls,
    # 7 solid x-min end, 8 solid x-max end
    def side(plane, cen):
        sid = np.full(cen.shape[0], plane + 1, dtype=np.int32)
        solid = cen[:, 1] < 0.0
        sid[(plane == 0) & solid] = 7
        sid[(plane == 1) & solid] = 8
        return sid
    m = box_mesh(nx, ny, nz, lo=(0.0, y0, 0.0), hi=(length, 1.0, 1.0), side_id=side,
                 axis_coords=(None, ys, None))
    cen_y = m.coord[m.intma - 1][:, :, 1].mean(axis=1)
    m.mat_elem = np.where(cen_y < 0.0, 1, 0).astype(np.int32)
    bc = {1: 508, 2: 520, 3: 532, 4: 530, 5: 530, 6: 530, 7: 530, 8: 530}
    kf = 1.0 / (re * pr)
    mats = {0: ("fluid", "fluid", 1.0, 1.0, kf, 1.0 / re, 0.0),
            1: ("solid", "solid", 1.0, 1.0, k_ratio * kf, 0.0, 0.0)}
    p = default_params(re=re, pr=pr, ntime=ntime, temp_calc=1, heat_flux_bc=q,
                       dimensional_mode=1, material_enabled=1, **over)
    return Case(mesh=m, bc_map=bc, params=p, materials=mats)
