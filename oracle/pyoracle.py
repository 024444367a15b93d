"""Test infrastructure only: ctypes binding of the C restatement (cbs_oracle.c)
and a reader for the reference harness dumps (ref_harness.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libcbs_oracle.so")
REF_HARNESS = os.path.join(HERE, "_ref", "cbs_ref_harness")
# the same harness with Step 2's pressure solve on the GPU drop-in (cbs3d_pcg_solve)
REF_GPU_HARNESS = os.path.join(HERE, "_ref", "cbs_ref_gpu_harness")


class OrcParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "solver_opt", "temp_calc", "transient_on", "dtfixed", "ilots", "htype", "cbs_scheme",
        "step2_check", "dtfix_end", "convection_type", "pnode",
        "dimensional_mode", "material_enabled", "massflow_enabled",
        "cg_precond", "cg_conv_test", "cg_max_iter")] + [("cinf", ctypes.c_double * 5)] + [
        (n, ctypes.c_double) for n in (
            "dtfix", "csafm", "csafm2", "epsilon1", "deltr", "re", "pr", "ri",
            "relToler", "absToler", "heat_flux_bc", "outlet_pressure_gauge",
            "inlet_mass_flow_rate", "inlet_density", "inlet_temperature",
            "inlet_u", "inlet_v", "inlet_w")]


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE, "_build/libcbs_oracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.POINTER(OrcParams), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                 ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        for fn in ("orc_step", "orc_time_step"):
            getattr(L, fn).argtypes = [ctypes.c_void_p, ctypes.c_int]
            getattr(L, fn).restype = ctypes.c_int
        for fn in ("orc_begin_step", "orc_lhs", "orc_step1", "orc_dt_correction", "orc_step2_rhs", "orc_solve_pressure",
                   "orc_step3", "orc_step4", "orc_convergence"):
            getattr(L, fn).argtypes = [ctypes.c_void_p]
            getattr(L, fn).restype = ctypes.c_int
        L.orc_pressure_multiply.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_get.restype = ctypes.c_long
        L.orc_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_long,
                              ctypes.c_char_p]
        L.orc_set.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_long]
        L.orc_error.restype = ctypes.c_char_p
        L.orc_error.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


def params_struct(p: dict) -> OrcParams:
    s = OrcParams()
    s.solver_opt = p["solver_opt"]; s.temp_calc = p["temp_calc"]; s.transient_on = p["transient_on"]
    s.dtfixed = p["dtfixed"]; s.ilots = p["ilots"]; s.htype = p["htype"]; s.cbs_scheme = p["cbs_scheme"]
    s.step2_check = p["step2_check"]; s.dtfix_end = p["dtfix_end"]
    s.convection_type = p["convection_type"]; s.pnode = p["pnode"]
    s.dimensional_mode = p["dimensional_mode"]; s.material_enabled = p["material_enabled"]
    s.massflow_enabled = p["massflow_enabled"]
    s.cg_precond = p["cg_precond"]; s.cg_conv_test = p["cg_conv_test"]; s.cg_max_iter = p["cg_max_iter"]
    for i, v in enumerate(p["cinf"]):
        s.cinf[i] = v
    s.dtfix = p["dtfix"]; s.csafm = p["csafm"]; s.csafm2 = p["csafm2"]; s.epsilon1 = p["epsilon1"]
    s.deltr = p["deltr"]; s.re = p["re"]; s.pr = p["pr"]; s.ri = p["ri"]
    s.relToler = p["relToler"]; s.absToler = p["absToler"]; s.heat_flux_bc = p["heat_flux_bc"]
    s.outlet_pressure_gauge = p["p_out"]; s.inlet_mass_flow_rate = p["mdot"]
    s.inlet_density = p["rho_in"]; s.inlet_temperature = p["T_in"]
    s.inlet_u = p["inlet_u"]; s.inlet_v = p["inlet_v"]; s.inlet_w = p["inlet_w"]
    return s


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def case_arrays(case):
    """Mesh arrays of a cases.Case in the layout orc_create expects."""
    m = case.mesh
    bf = np.ascontiguousarray(m.bfaces.copy())
    bf[:, 4] = np.vectorize(lambda r: case.bc_map[int(r)])(bf[:, 4]) if bf.size else bf[:, 4]
    mats = None
    if case.params.get("material_enabled", 0) > 0:
        props = np.array([case.materials[int(mid)][2:] for mid in m.mat_elem], dtype=np.float64)
        mats = [np.ascontiguousarray(props[:, i]) for i in range(5)]
    return (np.ascontiguousarray(m.intma, dtype=np.int32),
            np.ascontiguousarray(m.coord, dtype=np.float64), bf.astype(np.int32),
            np.ascontiguousarray(m.mat_elem, dtype=np.int32), mats)


class Oracle:
    """One oracle state built from a cases.Case."""

    def __init__(self, case):
        L = lib()
        self.case = case
        intma, coord, bf, mat, mats = case_arrays(case)
        self._keep = (intma, coord, bf, mat, mats)
        self.params = params_struct(case.params)
        err = ctypes.create_string_buffer(512)
        m = case.mesh
        args = [None] * 5 if mats is None else [_ptr(x) for x in mats]
        self.h = L.orc_create(ctypes.byref(self.params), m.nelem, m.npoin, m.nboun, _ptr(intma),
                              _ptr(coord), _ptr(bf), _ptr(mat), *args, err, 512)
        if not self.h:
            raise RuntimeError(err.value.decode())
        self.iitime = 0

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def _check(self, rc):
        if rc:
            raise RuntimeError(lib().orc_error(self.h).decode())

    def step(self, n: int = 1):
        for _ in range(n):
            self.iitime += 1
            self._check(lib().orc_step(self.h, self.iitime))

    def stage(self, name: str):
        L = lib()
        if name == "time_step":
            self._check(L.orc_time_step(self.h, self.iitime))
        else:
            self._check(getattr(L, "orc_" + name)(self.h))

    def get(self, name: str) -> np.ndarray:
        L = lib()
        t = ctypes.create_string_buffer(2)
        n = L.orc_get(self.h, name.encode(), None, 0, t)
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, dtype=np.float64 if t.value == b"d" else np.int32)
        L.orc_get(self.h, name.encode(), _ptr(out), n, t)
        return out

    def set(self, name: str, values):
        cur = self.get(name)
        a = np.ascontiguousarray(values, dtype=cur.dtype).ravel()
        if lib().orc_set(self.h, name.encode(), _ptr(a), a.size):
            raise KeyError(name)

    def pressure_multiply(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        lib().orc_pressure_multiply(self.h, _ptr(x), _ptr(y))
        return y


# ---------------------------------------------------------------------------
# reference harness dumps
# ---------------------------------------------------------------------------

def read_dump(directory: str) -> dict:
    out = {}
    with open(os.path.join(directory, "index.txt")) as f:
        for line in f:
            name, dt, n = line.split()
            out[name] = np.fromfile(os.path.join(directory, name + ".bin"),
                                    dtype=np.float64 if dt == "f8" else np.int32, count=int(n))
    return out


def run_reference(case_base: str, nsteps: int, outdir: str, stage: int = 0, every: int = 0,
                  threads: int = 1, gpu_pressure: bool = False) -> dict:
    os.makedirs(outdir, exist_ok=True)
    cmd = [REF_GPU_HARNESS if gpu_pressure else REF_HARNESS, case_base, str(nsteps), outdir]
    if stage:
        cmd += ["--stage", str(stage)]
    if every:
        cmd += ["--every", str(every)]
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    subprocess.run(cmd, check=True, env=env, stdout=subprocess.DEVNULL)
    return read_dump(outdir)
