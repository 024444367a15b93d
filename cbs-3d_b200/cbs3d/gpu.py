"""Python host of the B200 CBS3D engine: ctypes bindings of include/cbs3d_gpu.h.

The classes mirror the reference's host interface for the step path:

* ``Solver(case_name)`` with ``run()`` and ``state()`` stands for
  ``cbs::Solver`` (include/cbs/solver/Solver.hpp:25-51) and its run loop
  (src/solver/Solver.cpp:137-225).
* ``Context`` is one device-resident case; ``step()`` advances CBS steps
  (Solver::advanceOneStep, src/solver/Solver.cpp:609-680).
* ``PressureSolver`` is the solver_opt pressure-backend drop-in for
  ConjugateGradient::solvePressure (src/linalg/ConjugateGradient.cpp:584-869).

Errors raise ``CBSError`` carrying the C status code and the message worded
like the reference's std::runtime_error.  There is no CPU path: without the
built library every entry point raises.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG_ROOT, "libcbs3d_gpu.so")

FP64, MIXED = 0, 1

STATUS = {0: "OK", 1: "INVALID_INPUT", 2: "NOT_CONVERGED", 3: "BREAKDOWN", 4: "NONFINITE",
          5: "TIMEOUT", 6: "CUDA_ERROR", 7: "IO_ERROR", 8: "INTERNAL"}


class CBSError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{STATUS.get(code, code)}] {message}")
        self.code = code
        self.message = message


_i, _d = ctypes.c_int, ctypes.c_double


class Params(ctypes.Structure):
    _fields_ = [
        ("solver_opt", _i), ("restart_opt", _i), ("temp_calc", _i), ("cinf", _d * 5),
        ("ntime", _i), ("transient_on", _i), ("dtfixed", _i), ("dtfix", _d), ("iwrite", _i),
        ("csafm", _d), ("theta1", _d),
        ("cbs_scheme", _i), ("ilots", _i), ("htype", _i), ("step2_check", _i), ("rem_deltp", _i),
        ("beta_opt", _i), ("dtfix_end", _i), ("csafm2", _d), ("epsilon1", _d), ("deltr", _d),
        ("re", _d), ("pr", _d), ("ra", _d), ("ri", _d),
        ("convection_type", _i), ("pnode", _i), ("write_output", _i),
        ("write_time_output", _d), ("time_output_interval", _d), ("end_rtime", _d),
        ("relToler", _d), ("absToler", _d),
        ("vel_check", _i), ("l2norm_vel_tolerance", _d), ("temp_check", _i), ("l2norm_temp_tolerance", _d),
        ("paraview_output", _i), ("tecplot_output", _i), ("nusselt_calc", _i), ("nusselt_flag", _i),
        ("runtime_mod", _i),
        ("alpha_sf", _d), ("k_ratio", _d), ("source_solid", _d), ("heat_flux_bc", _d),
        ("dimensional_mode", _i), ("material_properties_enabled", _i), ("mass_flow_inlet_enabled", _i),
        ("p_ref", _d), ("model_depth", _d), ("inlet_mass_flow_rate", _d), ("inlet_density", _d),
        ("inlet_temperature", _d), ("outlet_pressure_gauge", _d),
        ("inlet_u", _d), ("inlet_v", _d), ("inlet_w", _d),
        ("nusselt_Tinf", _d), ("nusselt_Tref", _d), ("nusselt_diameter", _d),
        ("cg_preconditioner", _i), ("cg_conv_test", _i), ("cg_max_iter", _i), ("l2norm_pres_tolerance", _d),
        ("residual_log_enabled", _i), ("residual_log_every", _i), ("console_log_every", _i),
        ("live_residual_plot", _i), ("vtu_output_enabled", _i), ("vtu_output_every_iterations", _i),
        ("vtu_output_every_sim_time", _d),
        ("write_boundary_debug_arrays", _i), ("steady_min_iterations", _i), ("art_diff", _i),
    ]


class Mesh(ctypes.Structure):
    _fields_ = [("nelem", _i), ("npoin", _i), ("nboun", _i),
                ("intma", ctypes.c_void_p), ("coord", ctypes.c_void_p), ("bface", ctypes.c_void_p),
                ("mat_elem", ctypes.c_void_p), ("rho", ctypes.c_void_p), ("cp", ctypes.c_void_p),
                ("k", ctypes.c_void_p), ("mu", ctypes.c_void_p), ("qvol", ctypes.c_void_p)]


class Options(ctypes.Structure):
    _fields_ = [("precision", _i), ("device", _i), ("inner_tol", _d), ("use_graph", _i),
                ("pcg_blocks", _i), ("verbose", _i), ("time_pcg", _i), ("pcg_kernel", _i), ("case_cache", _i),
                ("pcg_two_level", _i), ("pcg_multigrid", _i)]


class CGResult(ctypes.Structure):
    _fields_ = [("iterations", _i), ("initial_l2", _d), ("final_l2", _d), ("final_relative_l2", _d),
                ("final_max_abs", _d), ("converged", _i),
                ("total_seconds", _d), ("setup_seconds", _d), ("matvec_seconds", _d), ("dot_seconds", _d),
                ("preconditioner_seconds", _d), ("vector_update_seconds", _d), ("constraint_seconds", _d),
                ("matvec_calls", _i), ("dot_calls", _i), ("preconditioner_calls", _i), ("outer_sweeps", _i)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class StepStats(ctypes.Structure):
    _fields_ = [("steps_done", _i), ("iitime", _i), ("failed_step", _i), ("dtreal", _d), ("rtime", _d),
                ("cg", CGResult), ("cg_iterations_total", ctypes.c_longlong), ("hb", _d * 15),
                ("gpu_seconds", _d), ("steady_reached", _i), ("pcg_seconds", _d), ("pcg_launches", _i),
                ("kernel_launches", ctypes.c_longlong), ("pcg_bytes_per_iter", _d),
                ("pcg_kernel", _i)]


class BatchOptions(ctypes.Structure):
    _fields_ = [("base", Options), ("autotune", _i), ("rows_per_thread", _i), ("spread", _i)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("instances", _i), ("waves", _i), ("rows_per_thread", _i), ("spread", _i), ("mixed_waves", _i),
                ("tuned", _i), ("candidates", _i), ("cand_rows", _i * 8), ("cand_spread", _i * 8),
                ("cand_ms", _d * 8)]


# case-generator parameter names -> cbs3d_params fields
_PAR_MAP = {
    "l2v": "l2norm_vel_tolerance", "l2T": "l2norm_temp_tolerance", "paraview": "paraview_output",
    "tecplot": "tecplot_output", "material_enabled": "material_properties_enabled",
    "massflow_enabled": "mass_flow_inlet_enabled", "mdot": "inlet_mass_flow_rate", "rho_in": "inlet_density",
    "T_in": "inlet_temperature", "p_out": "outlet_pressure_gauge", "Tinf": "nusselt_Tinf",
    "Tref": "nusselt_Tref", "Dnu": "nusselt_diameter", "cg_precond": "cg_preconditioner",
    "l2p": "l2norm_pres_tolerance", "reslog": "residual_log_enabled", "reslog_every": "residual_log_every",
    "console_every": "console_log_every", "live_plot": "live_residual_plot", "vtu": "vtu_output_enabled",
    "vtu_every": "vtu_output_every_iterations", "vtu_time": "vtu_output_every_sim_time",
    "dbg_arrays": "write_boundary_debug_arrays", "steady_min": "steady_min_iterations",
}

_lib = None


def lib():
    """Loads libcbs3d_gpu.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise CBSError(8, f"CUDA engine not built: {LIB_PATH} is missing (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        vp, cp = ctypes.c_void_p, ctypes.c_char_p
        L.cbs3d_default_params.argtypes = [ctypes.POINTER(Params)]
        L.cbs3d_default_options.argtypes = [ctypes.POINTER(Options)]
        L.cbs3d_status_string.restype = cp
        L.cbs3d_create.argtypes = [ctypes.POINTER(Mesh), ctypes.POINTER(Params), ctypes.POINTER(Options),
                                   ctypes.POINTER(vp), cp, ctypes.c_size_t]
        L.cbs3d_create_from_case.argtypes = [cp, ctypes.POINTER(Options), ctypes.POINTER(vp), cp, ctypes.c_size_t]
        L.cbs3d_read_params.argtypes = [cp, ctypes.POINTER(Params), ctypes.POINTER(_i), ctypes.POINTER(_i),
                                        ctypes.POINTER(_i), cp, ctypes.c_size_t]
        L.cbs3d_destroy.argtypes = [vp]
        L.cbs3d_last_error.argtypes = [vp]
        L.cbs3d_last_error.restype = cp
        L.cbs3d_step.argtypes = [vp, _i, _i, ctypes.POINTER(StepStats)]
        L.cbs3d_upload_fields.argtypes = [vp, vp, vp, vp]
        L.cbs3d_download_fields.argtypes = [vp, vp, vp, vp]
        L.cbs3d_get_array.argtypes = [vp, cp, vp, ctypes.c_long, ctypes.POINTER(ctypes.c_long)]
        L.cbs3d_set_array.argtypes = [vp, cp, vp, ctypes.c_long]
        L.cbs3d_run_stage.argtypes = [vp, cp]
        L.cbs3d_pressure_multiply.argtypes = [vp, vp, vp]
        L.cbs3d_pcg_create.argtypes = [_i, _i, vp, vp, _i, vp, vp, ctypes.POINTER(Options), ctypes.POINTER(vp),
                                       cp, ctypes.c_size_t]
        L.cbs3d_pcg_solve.argtypes = [vp, _i, _i, _i, _d, _d, vp, vp, vp, vp, ctypes.POINTER(CGResult)]
        L.cbs3d_pcg_destroy.argtypes = [vp]
        L.cbs3d_pcg_last_error.argtypes = [vp]
        L.cbs3d_pcg_last_error.restype = cp
        L.cbs3d_case_digest.argtypes = [cp, _i, ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(_i), cp,
                                        ctypes.c_size_t]
        L.cbs3d_case_digest.restype = _i
        L.cbs3d_write_vtu_case.argtypes = [cp, cp, vp, vp, vp, cp, ctypes.c_size_t]
        L.cbs3d_write_vtu_case.restype = _i
        L.cbs3d_write_vtu.argtypes = [vp, cp]
        L.cbs3d_write_vtu.restype = _i
        L.cbs3d_write_vtu_async.argtypes = [vp, cp]
        L.cbs3d_write_vtu_async.restype = _i
        L.cbs3d_vtu_flush.argtypes = [vp]
        L.cbs3d_vtu_flush.restype = _i
        L.cbs3d_write_residual_rows.argtypes = [vp, cp, _i]
        L.cbs3d_write_residual_rows.restype = _i
        L.cbs3d_step_history.argtypes = [vp, _i, _i, vp]
        L.cbs3d_step_history.restype = _i
        L.cbs3d_solve_pressure.argtypes = [vp, vp, vp, vp, vp, ctypes.POINTER(CGResult)]
        L.cbs3d_solve_pressure.restype = _i
        L.cbs3d_set_body_force.argtypes = [vp, vp]
        L.cbs3d_objective_run.argtypes = [vp, _i, vp, ctypes.POINTER(_d)]
        L.cbs3d_tlm_run.argtypes = [vp, _i, vp, vp, ctypes.POINTER(_d), ctypes.POINTER(_d)]
        L.cbs3d_adjoint_run.argtypes = [vp, _i, _i, vp, ctypes.POINTER(_d), vp]
        L.cbs3d_heat_flux_face_count.argtypes = [vp, ctypes.POINTER(_i)]
        L.cbs3d_set_face_heat_flux.argtypes = [vp, vp]
        L.cbs3d_heat_objective_run.argtypes = [vp, _i, vp, ctypes.POINTER(_d)]
        L.cbs3d_heat_tlm_run.argtypes = [vp, _i, vp, vp, ctypes.POINTER(_d), ctypes.POINTER(_d)]
        L.cbs3d_heat_adjoint_run.argtypes = [vp, _i, _i, vp, ctypes.POINTER(_d), vp]
        L.cbs3d_default_batch_options.argtypes = [ctypes.POINTER(BatchOptions)]
        L.cbs3d_batch_create.argtypes = [_i, ctypes.POINTER(Mesh), ctypes.POINTER(Params),
                                         ctypes.POINTER(BatchOptions), ctypes.POINTER(vp), cp, ctypes.c_size_t]
        L.cbs3d_batch_step.argtypes = [vp, _i, ctypes.POINTER(StepStats), ctypes.POINTER(_d)]
        L.cbs3d_batch_download_fields.argtypes = [vp, _i, vp, vp, vp]
        L.cbs3d_batch_get_info.argtypes = [vp, ctypes.POINTER(BatchInfo)]
        L.cbs3d_batch_destroy.argtypes = [vp]
        L.cbs3d_batch_last_error.argtypes = [vp]
        L.cbs3d_batch_last_error.restype = cp
        L.cbs3d_selftest_wait_timeout.argtypes = [_i, ctypes.POINTER(_i)]
        L.cbs3d_selftest_wait_timeout.restype = _i
        L.cbs3d_coarse_inverse.argtypes = [_i, _i, vp, vp, _i]
        L.cbs3d_coarse_inverse.restype = _i
        for fn in ("cbs3d_create", "cbs3d_create_from_case", "cbs3d_read_params", "cbs3d_step",
                   "cbs3d_upload_fields", "cbs3d_download_fields", "cbs3d_get_array", "cbs3d_set_array",
                   "cbs3d_run_stage", "cbs3d_pressure_multiply", "cbs3d_pcg_create", "cbs3d_pcg_solve",
                   "cbs3d_set_body_force", "cbs3d_objective_run", "cbs3d_tlm_run", "cbs3d_adjoint_run",
                   "cbs3d_heat_flux_face_count", "cbs3d_set_face_heat_flux", "cbs3d_heat_objective_run",
                   "cbs3d_heat_tlm_run", "cbs3d_heat_adjoint_run",
                   "cbs3d_batch_create", "cbs3d_batch_step", "cbs3d_batch_download_fields", "cbs3d_batch_get_info"):
            getattr(L, fn).restype = _i
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def make_params(p: dict) -> Params:
    s = Params()
    lib().cbs3d_default_params(ctypes.byref(s))
    names = {f for f, _ in Params._fields_}
    for key, val in p.items():
        field = _PAR_MAP.get(key, key)
        if field == "cinf":
            for i, v in enumerate(val):
                s.cinf[i] = v
        elif field in names:
            setattr(s, field, val)
    return s


def case_digest(case_name: str, use_cache: bool = False):
    """(digest, from_cache) of a case's parsed inputs -- host only, no GPU."""
    d, hit = ctypes.c_ulonglong(), _i()
    err = ctypes.create_string_buffer(1024)
    rc = lib().cbs3d_case_digest(case_name.encode(), 1 if use_cache else 0, ctypes.byref(d), ctypes.byref(hit),
                                 err, 1024)
    if rc != 0:
        raise CBSError(rc, err.value.decode())
    return d.value, bool(hit.value)


def make_options(precision: int = FP64, device: int = 0, inner_tol: float = 0.05, use_graph: bool = True,
                 pcg_blocks: int = 0, time_pcg: bool = False, pcg_kernel: int = 0) -> Options:
    o = Options()
    lib().cbs3d_default_options(ctypes.byref(o))
    o.precision = precision
    o.device = device
    o.inner_tol = inner_tol
    o.use_graph = 1 if use_graph else 0
    o.pcg_blocks = pcg_blocks
    o.time_pcg = 1 if time_pcg else 0
    o.pcg_kernel = pcg_kernel
    return o


def _mesh_params(case):
    """cbs3d_mesh and cbs3d_params of a generated case, plus the arrays they
    point into (kept alive by the caller)."""
    m = case.mesh
    bf = np.ascontiguousarray(m.bfaces.copy())
    if bf.size:
        lut = np.zeros(int(bf[:, 4].max()) + 1, dtype=np.int32)
        for raw, bc in case.bc_map.items():
            if raw < lut.size:
                lut[raw] = bc
        bf[:, 4] = lut[bf[:, 4]]
    bf = np.ascontiguousarray(bf.astype(np.int32))
    intma = np.ascontiguousarray(m.intma, dtype=np.int32)
    coord = np.ascontiguousarray(m.coord, dtype=np.float64)
    mat = np.ascontiguousarray(m.mat_elem, dtype=np.int32)
    props = [None] * 5
    if case.params.get("material_enabled", 0) > 0:
        pr = np.array([case.materials[int(mid)][2:] for mid in m.mat_elem], dtype=np.float64)
        props = [np.ascontiguousarray(pr[:, i]) for i in range(5)]
    mesh = Mesh(m.nelem, m.npoin, m.nboun, _ptr(intma), _ptr(coord), _ptr(bf), _ptr(mat),
                *[_ptr(x) for x in props])
    return mesh, make_params(case.params), (intma, coord, bf, mat, props)


class Context:
    """One case resident on the GPU."""

    def __init__(self, case=None, case_name: str | None = None, precision: int = FP64, device: int = 0,
                 inner_tol: float = 0.05, use_graph: bool = True, pcg_blocks: int = 0, time_pcg: bool = False,
                 pcg_kernel: int = 0, case_cache: bool = False, two_level: bool = False,
                 multigrid: bool = False):
        L = lib()
        self.h = ctypes.c_void_p()
        self.device = device
        err = ctypes.create_string_buffer(1024)
        opt = make_options(precision, device, inner_tol, use_graph, pcg_blocks, time_pcg, pcg_kernel)
        opt.case_cache = 1 if case_cache else 0
        opt.pcg_two_level = 1 if two_level else 0
        opt.pcg_multigrid = 1 if multigrid else 0
        if case_name is not None:
            rc = L.cbs3d_create_from_case(case_name.encode(), ctypes.byref(opt), ctypes.byref(self.h), err, 1024)
        else:
            mesh, par, self._keep = _mesh_params(case)
            rc = L.cbs3d_create(ctypes.byref(mesh), ctypes.byref(par), ctypes.byref(opt), ctypes.byref(self.h),
                                err, 1024)
        if rc != 0:
            self.h = None
            raise CBSError(rc, err.value.decode())
        self.npoin = self._get_len("pres")
        self.nelem = self._get_len("delte")

    def close(self):
        if getattr(self, "h", None):
            lib().cbs3d_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc: int):
        if rc != 0:
            raise CBSError(rc, lib().cbs3d_last_error(self.h).decode())

    def write_vtu(self, path: str):
        """VTU snapshot of the current fields (Post::writeVTU), written now."""
        self._check(lib().cbs3d_write_vtu(self.h, path.encode()))

    def write_vtu_async(self, path: str):
        """The same snapshot, taken on the device and written by a host
        thread while later steps run; vtu_flush() waits for the files."""
        self._check(lib().cbs3d_write_vtu_async(self.h, path.encode()))

    def vtu_flush(self):
        self._check(lib().cbs3d_vtu_flush(self.h))

    def _get_len(self, name: str) -> int:
        n = ctypes.c_long(0)
        self._check(lib().cbs3d_get_array(self.h, name.encode(), None, 0, ctypes.byref(n)))
        return n.value

    def step(self, n: int = 1, stop_on_steady: bool = False) -> StepStats:
        st = StepStats()
        self._check(lib().cbs3d_step(self.h, n, 1 if stop_on_steady else 0, ctypes.byref(st)))
        return st

    def stage(self, name: str):
        self._check(lib().cbs3d_run_stage(self.h, name.encode()))

    def get(self, name: str) -> np.ndarray:
        n = self._get_len(name)
        ints = name in ("fedge", "iside", "color_ptr", "color_elem", "bc_list", "wall_node_list", "ncolor")
        out = np.empty(n, dtype=np.int32 if ints else np.float64)
        self._check(lib().cbs3d_get_array(self.h, name.encode(), _ptr(out), n, None))
        return out

    def set(self, name: str, values):
        a = np.ascontiguousarray(values, dtype=np.float64).ravel()
        self._check(lib().cbs3d_set_array(self.h, name.encode(), _ptr(a), a.size))

    def fields(self):
        u = np.empty(3 * self.npoin)
        p = np.empty(self.npoin)
        t = np.empty(self.npoin)
        self._check(lib().cbs3d_download_fields(self.h, _ptr(u), _ptr(p), _ptr(t)))
        return u, p, t

    def upload(self, u=None, p=None, t=None):
        arrs = [None if x is None else np.ascontiguousarray(x, dtype=np.float64) for x in (u, p, t)]
        self._check(lib().cbs3d_upload_fields(self.h, *[_ptr(a) for a in arrs]))

    # ---- body force, tangent-linear and adjoint runs (extension)
    def set_body_force(self, f=None):
        """f[3*npoin] node-major, or None to remove it."""
        a = None if f is None else np.ascontiguousarray(f, dtype=np.float64).reshape(-1)
        if a is not None and a.size != 3 * self.npoin:
            raise ValueError("body force must have 3*npoin entries")
        self._bf = a
        self._check(lib().cbs3d_set_body_force(self.h, _ptr(a)))

    def objective(self, nsteps: int, w) -> float:
        """J = 1/2 sum w_i |u_i|^2 after nsteps steps; the state is restored."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        J = ctypes.c_double()
        self._check(lib().cbs3d_objective_run(self.h, nsteps, _ptr(w), ctypes.byref(J)))
        return J.value

    def tlm(self, nsteps: int, w, df):
        """(J, dJ/df . df) from the tangent-linear model; the state is restored."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        df = np.ascontiguousarray(df, dtype=np.float64).reshape(-1)
        J, dJ = ctypes.c_double(), ctypes.c_double()
        self._check(lib().cbs3d_tlm_run(self.h, nsteps, _ptr(w), _ptr(df), ctypes.byref(J), ctypes.byref(dJ)))
        return J.value, dJ.value

    def adjoint(self, nsteps: int, w, every: int = 20):
        """(J, dJ/df[3*npoin]) with checkpoints every `every` steps; the state is restored."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        g = np.empty(3 * self.npoin)
        J = ctypes.c_double()
        self._check(lib().cbs3d_adjoint_run(self.h, nsteps, every, _ptr(w), ctypes.byref(J), _ptr(g)))
        return J.value, g

    def heat_flux_faces(self) -> int:
        n = _i()
        self._check(lib().cbs3d_heat_flux_face_count(self.h, ctypes.byref(n)))
        return n.value

    def set_face_heat_flux(self, q=None):
        """Per-face heat flux on the BC-532 faces, or None for the uniform value."""
        a = None if q is None else np.ascontiguousarray(q, dtype=np.float64)
        self._q = a
        self._check(lib().cbs3d_set_face_heat_flux(self.h, _ptr(a)))

    def heat_objective(self, nsteps: int, w) -> float:
        """J = sum w_i T_i after nsteps steps; the state is restored."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        J = ctypes.c_double()
        self._check(lib().cbs3d_heat_objective_run(self.h, nsteps, _ptr(w), ctypes.byref(J)))
        return J.value

    def heat_tlm(self, nsteps: int, w, dq):
        w = np.ascontiguousarray(w, dtype=np.float64)
        dq = np.ascontiguousarray(dq, dtype=np.float64)
        J, dJ = ctypes.c_double(), ctypes.c_double()
        self._check(lib().cbs3d_heat_tlm_run(self.h, nsteps, _ptr(w), _ptr(dq), ctypes.byref(J), ctypes.byref(dJ)))
        return J.value, dJ.value

    def heat_adjoint(self, nsteps: int, w, every: int = 20):
        """(J, dJ/dq[faces]) with checkpoints every `every` steps; the state is restored."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        g = np.empty(self.heat_flux_faces())
        J = ctypes.c_double()
        self._check(lib().cbs3d_heat_adjoint_run(self.h, nsteps, every, _ptr(w), ctypes.byref(J), _ptr(g)))
        return J.value, g

    def solve_pressure(self, gstif, pdiag, rhs1, pres):
        """cbs3d_solve_pressure on copies: returns (pres, rhs1, pdiag, result dict)."""
        g = np.ascontiguousarray(gstif, dtype=np.float64)
        pd, r1, p = (np.array(a, dtype=np.float64) for a in (pdiag, rhs1, pres))
        res = CGResult()
        rc = lib().cbs3d_solve_pressure(self.h, _ptr(g), _ptr(pd), _ptr(r1), _ptr(p), ctypes.byref(res))
        if rc != 0 and rc != 2:
            self._check(rc)
        out = res.as_dict()
        out["status"] = rc
        return p, r1, pd, out

    def pressure_multiply(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        self._check(lib().cbs3d_pressure_multiply(self.h, _ptr(x), _ptr(y)))
        return y


def selftest_wait_timeout(device: int = 0) -> int:
    """Runs the bounded-wait self-test; returns the status the device recorded."""
    obs = _i(0)
    rc = lib().cbs3d_selftest_wait_timeout(device, ctypes.byref(obs))
    if rc != 0:
        raise CBSError(rc, "selftest launch failed")
    return obs.value


def coarse_inverse(a, variant: int = 0, device: int = 0) -> np.ndarray:
    """Inverse of a small dense SPD matrix by the two-level preconditioner's
    device Gauss-Jordan kernel (variant 0: register tiles, 1: shared memory)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.ndim != 2 or a.shape[0] != a.shape[1]:
        raise ValueError("square matrix expected")
    out = np.empty_like(a)
    rc = lib().cbs3d_coarse_inverse(device, a.shape[0], _ptr(a), _ptr(out), variant)
    if rc != 0:
        raise CBSError(rc, "coarse inverse failed")
    return out


class PressureSolver:
    """Drop-in for ConjugateGradient::solvePressure on the GPU."""

    def __init__(self, intma, mat_elem, bc_list, bc_values, precision: int = FP64, device: int = 0,
                 inner_tol: float = 0.05, multigrid: bool = False):
        L = lib()
        self.h = ctypes.c_void_p()
        intma = np.ascontiguousarray(intma, dtype=np.int32).reshape(-1)
        mat = None if mat_elem is None else np.ascontiguousarray(mat_elem, dtype=np.int32)
        bl = np.ascontiguousarray(bc_list, dtype=np.int32)
        bv = np.ascontiguousarray(bc_values, dtype=np.float64)
        self.nelem = intma.size // 4
        self.npoin = int(intma.max())
        err = ctypes.create_string_buffer(1024)
        opt = make_options(precision, device, inner_tol)
        opt.pcg_multigrid = 1 if multigrid else 0
        rc = L.cbs3d_pcg_create(self.nelem, self.npoin, _ptr(intma), _ptr(mat), bl.size, _ptr(bl), _ptr(bv),
                                ctypes.byref(opt), ctypes.byref(self.h), err, 1024)
        if rc != 0:
            self.h = None
            raise CBSError(rc, err.value.decode())

    def solve(self, gstif, pdiag, rhs1, pres, cg_preconditioner=1, cg_conv_test=2, cg_max_iter=100000,
              relToler=1e-10, absToler=1e-300):
        """Solves in place on copies; returns (pres, rhs1, pdiag, result dict)."""
        g = np.ascontiguousarray(gstif, dtype=np.float64)
        pd = np.array(pdiag, dtype=np.float64)
        r1 = np.array(rhs1, dtype=np.float64)
        p = np.array(pres, dtype=np.float64)
        res = CGResult()
        rc = lib().cbs3d_pcg_solve(self.h, cg_preconditioner, cg_conv_test, cg_max_iter, relToler, absToler,
                                   _ptr(g), _ptr(pd), _ptr(r1), _ptr(p), ctypes.byref(res))
        if rc != 0 and rc != 2:
            raise CBSError(rc, lib().cbs3d_pcg_last_error(self.h).decode())
        out = res.as_dict()
        out["status"] = rc
        return p, r1, pd, out

    def close(self):
        if getattr(self, "h", None):
            lib().cbs3d_pcg_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class Solver:
    """cbs::Solver over the GPU engine: reads <case>.par/.plt/.bco, then run()
    loops steps until ntime or the reference's stop tests."""

    def __init__(self, case_name: str, precision: int = FP64, device: int = 0):
        self.case_name = case_name
        self.ctx = Context(case_name=case_name, precision=precision, device=device)
        par = Params()
        ne, npn, nb = _i(), _i(), _i()
        err = ctypes.create_string_buffer(1024)
        rc = lib().cbs3d_read_params(case_name.encode(), ctypes.byref(par), ctypes.byref(ne), ctypes.byref(npn),
                                     ctypes.byref(nb), err, 1024)
        if rc != 0:
            raise CBSError(rc, err.value.decode())
        self.params = par
        self.history = []

    def run(self, chunk: int = 50):
        left = self.params.ntime
        while left > 0:
            st = self.ctx.step(min(chunk, left), stop_on_steady=True)
            self.history.append(st)
            left -= st.steps_done
            if st.steady_reached:
                break
        return self.history[-1] if self.history else None

    def state(self) -> dict:
        u, p, t = self.ctx.fields()
        return {"unkno": u.reshape(-1, 3), "pres": p, "temperature": t}


class Batch:
    """Many independent cases advanced together (cbs3d_batch_*): one CUDA
    graph per step, the pressure systems solved by one cooperative launch
    per wave of instances."""

    def __init__(self, cases, precision: int = FP64, device: int = 0, autotune: bool = True,
                 rows_per_thread: int = 4, spread: bool = True, use_graph: bool = True, inner_tol: float = 0.05):
        L = lib()
        self.h = ctypes.c_void_p()
        self.n = len(cases)
        opt = BatchOptions()
        L.cbs3d_default_batch_options(ctypes.byref(opt))
        opt.base = make_options(precision, device, inner_tol, use_graph)
        opt.autotune = 1 if autotune else 0
        opt.rows_per_thread = rows_per_thread
        opt.spread = 1 if spread else 0
        meshes = (Mesh * self.n)()
        pars = (Params * self.n)()
        self._keep = []
        self.npoin = []
        for i, c in enumerate(cases):
            m, p, keep = _mesh_params(c)
            meshes[i] = m
            pars[i] = p
            self._keep.append(keep)
            self.npoin.append(c.mesh.npoin)
        err = ctypes.create_string_buffer(1024)
        rc = L.cbs3d_batch_create(self.n, meshes, pars, ctypes.byref(opt), ctypes.byref(self.h), err, 1024)
        if rc != 0:
            self.h = None
            raise CBSError(rc, err.value.decode())

    def _check(self, rc: int):
        if rc != 0:
            raise CBSError(rc, lib().cbs3d_batch_last_error(self.h).decode())

    def step(self, n: int = 1):
        """n steps of every instance; returns (per-instance StepStats, device seconds)."""
        st = (StepStats * self.n)()
        sec = ctypes.c_double()
        self._check(lib().cbs3d_batch_step(self.h, n, st, ctypes.byref(sec)))
        return list(st), sec.value

    def fields(self, i: int):
        N = self.npoin[i]
        u, p, t = np.empty(3 * N), np.empty(N), np.empty(N)
        self._check(lib().cbs3d_batch_download_fields(self.h, i, _ptr(u), _ptr(p), _ptr(t)))
        return u, p, t

    def info(self) -> dict:
        inf = BatchInfo()
        self._check(lib().cbs3d_batch_get_info(self.h, ctypes.byref(inf)))
        d = {n: getattr(inf, n) for n, _ in BatchInfo._fields_ if not n.startswith("cand_")}
        d["candidates_timed"] = [(inf.cand_rows[k], inf.cand_spread[k], inf.cand_ms[k]) for k in range(inf.candidates)]
        return d

    def close(self):
        if getattr(self, "h", None):
            lib().cbs3d_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
