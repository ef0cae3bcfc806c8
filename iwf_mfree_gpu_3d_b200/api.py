"""Python binding of libmfree.so (include/mfree.h) over ctypes.

The reference drives its step from C++ (src/mfree_gpu_3d.cpp:75-218): it builds
a ``particle_gpu`` from host arrays, uploads the constant records with
``actions_setup_*`` / ``interactions_setup_*``, creates the locked grid, the
blanking box and the tools, then calls ``leap_frog::step`` once per time step.
``Simulation`` mirrors those calls one to one on top of the C ABI; every call
raises ``MfreeError`` on a non-zero status.  There is no CPU fallback: if the
CUDA library cannot be loaded, construction fails.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libmfree.so")

FIELDS = ["POS", "VEL", "VEL_BC", "H", "RHO", "P", "S", "R", "FC", "FT", "NRM", "FIXED", "BLANKED",
          "TOOL_PARTICLE", "EPS_PL", "EPS_PL_DOT", "T", "POS_T", "VEL_T", "RHO_T", "S_T", "T_T", "NUM_NBH",
          "IDX", "HASH", "ID", "POS_HALF"]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}
INT_FIELDS = {"NUM_NBH", "IDX", "HASH", "ID"}

COND_NONE, COND_BROOKSHAW, COND_PSE = 0, 1, 2
CONTACT_HASHED, CONTACT_EXHAUSTIVE = 0, 1

# every symbol include/mfree.h declares
EXPORTS = [
    "mfree_create", "mfree_destroy", "mfree_last_error", "mfree_set_physics", "mfree_set_correctors",
    "mfree_set_johnson_cook", "mfree_set_thermal_workpiece", "mfree_set_thermal_tool", "mfree_set_options",
    "mfree_get_options", "mfree_set_grid", "mfree_set_grid_velocity", "mfree_set_grid_adaptive", "mfree_set_blanking", "mfree_set_time",
    "mfree_get_time", "mfree_add_tool", "mfree_tool_set_birth_death", "mfree_get_tool_forces",
    "mfree_get_tool_info", "mfree_get_tool_normals", "mfree_get_tool_cells", "mfree_step", "mfree_advance",
    "mfree_sync", "mfree_get_counts", "mfree_field_width", "mfree_get_field", "mfree_set_field",
    "mfree_get_field_f64", "mfree_get_cells", "mfree_get_grid", "mfree_get_counters", "mfree_read_mesh_json",
    "mfree_read_mesh_ldynak", "mfree_read_mesh_ldynak_quad", "mfree_free", "mfree_set_kernel_timing", "mfree_get_kernel_times",
    "mfree_probe_fp32_peak", "mfree_timer_start", "mfree_timer_stop", "mfree_set_device",
    "mfree_cell_list_static", "mfree_batch_create", "mfree_batch_destroy", "mfree_batch_admit", "mfree_batch_step",
    "mfree_batch_query", "mfree_batch_context", "mfree_batch_retire", "mfree_batch_info", "mfree_batch_set_tiling",
    "mfree_batch_get_tiling", "mfree_batch_autotune", "mfree_batch_sync", "mfree_batch_timer_start",
    "mfree_batch_timer_stop", "mfree_device_bytes", "mfree_scene_bytes", "mfree_write_vtk", "mfree_output_wait",
    "mfree_write_vtk_tools", "mfree_write_vtk_blanking", "mfree_append_force_log", "mfree_export_state",
    "mfree_import_state", "mfree_inject_fault", "mfree_get_array", "mfree_set_array", "mfree_array_device_ptr",
    "mfree_bounds_checked", "mfree_get_energies",
]
ARRAYS = ["POS_H", "VEL_RHO", "S_A", "S_B", "POS_T", "VEL_T", "S_T_A", "S_T_B", "FC", "FT", "VEL_BC", "LO", "LO_B"]
ERR_ARG = -1
ERR_BUDGET = -7
ERR_TIMEOUT = -8
KERNELS = ["clock", "hash", "scan_reduce", "scan_top", "scan_down", "scatter", "cell_fixup", "gather_predict",
           "interact", "finalize", "force_final"]


class MfreeError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"mfree status {status}: {msg}")
        self.status = status


class Phys(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("E", "nu", "rho0", "K", "G", "mass")]


class Trml(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("cp", "tq", "k", "alpha", "T_init", "eta")]


class Corr(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("wdeltap", "stresseps", "xspheps", "alpha", "beta", "eta")]


class Joco(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("A", "B", "C", "n", "m", "Tmelt", "Tref", "eps_dot_ref", "clamp_temp")]


class Options(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("cspm", "conduction", "precision", "max_secant_iter",
                                       "lanes_per_particle", "diagnostics", "friction_tool_vel",
                                       "tile_depth", "full_stencil")]


class Counters(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("steps", "secant_failures", "out_of_grid", "contact_search_cap",
                                         "nan_blanked", "staging_timeouts", "full_stencil_steps",
                                         "bounds_errors", "pse_zero_targets")]


_lib = None


def lib(path: str = LIB_PATH):
    """Load libmfree.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with python -m iwf_mfree_gpu_3d_b200.build")
    L = C.CDLL(path)
    I, F, P = C.c_int, C.c_float, C.c_void_p
    fp = C.POINTER(C.c_float)
    ip = C.POINTER(C.c_int)
    L.mfree_last_error.restype = C.c_char_p
    L.mfree_create.argtypes = [I, fp, fp, fp, fp, fp, fp, fp, P, C.POINTER(P)]
    L.mfree_destroy.argtypes = [P]
    L.mfree_set_physics.argtypes = [P, C.POINTER(Phys)]
    L.mfree_set_correctors.argtypes = [P, C.POINTER(Corr)]
    L.mfree_set_johnson_cook.argtypes = [P, C.POINTER(Joco)]
    L.mfree_set_thermal_workpiece.argtypes = [P, C.POINTER(Trml)]
    L.mfree_set_thermal_tool.argtypes = [P, C.POINTER(Trml)]
    L.mfree_set_options.argtypes = [P, C.POINTER(Options)]
    L.mfree_get_options.argtypes = [P, C.POINTER(Options)]
    L.mfree_set_grid.argtypes = [P, fp, fp, F]
    L.mfree_set_grid_velocity.argtypes = [P, fp]
    L.mfree_set_grid_adaptive.argtypes = [P, C.c_long]
    L.mfree_get_array.argtypes = [P, I, fp]
    L.mfree_get_energies.argtypes = [P, C.POINTER(C.c_double)]
    L.mfree_set_array.argtypes = [P, I, fp]
    L.mfree_array_device_ptr.argtypes = [P, I, C.POINTER(P)]
    L.mfree_set_blanking.argtypes = [P, fp, fp, fp, F]
    L.mfree_set_time.argtypes = [P, F, F]
    L.mfree_get_time.argtypes = [P, fp, fp]
    L.mfree_add_tool.argtypes = [P, fp, I, ip, I, fp, F, F, I, ip]
    L.mfree_tool_set_birth_death.argtypes = [P, I, F, F]
    L.mfree_get_tool_forces.argtypes = [P, fp]
    L.mfree_get_tool_info.argtypes = [P, I, ip, ip, ip, fp, fp, fp]
    L.mfree_get_tool_normals.argtypes = [P, I, fp]
    L.mfree_get_tool_cells.argtypes = [P, I, ip, ip]
    L.mfree_step.argtypes = [P, I]
    L.mfree_advance.argtypes = [P, I, I, I]
    L.mfree_sync.argtypes = [P]
    L.mfree_get_counts.argtypes = [P, ip, ip]
    L.mfree_field_width.argtypes = [I]
    L.mfree_get_field.argtypes = [P, I, P]
    L.mfree_set_field.argtypes = [P, I, P]
    L.mfree_get_field_f64.argtypes = [P, I, C.POINTER(C.c_double)]
    L.mfree_get_cells.argtypes = [P, ip, ip]
    L.mfree_get_grid.argtypes = [P, C.POINTER(C.c_long), C.POINTER(C.c_long), C.POINTER(C.c_long), fp, fp]
    L.mfree_get_counters.argtypes = [P, C.POINTER(Counters)]
    L.mfree_read_mesh_json.argtypes = [C.c_char_p, C.POINTER(fp), ip, C.POINTER(ip), ip]
    L.mfree_read_mesh_ldynak.argtypes = [C.c_char_p, C.POINTER(fp), ip, C.POINTER(ip), ip]
    L.mfree_read_mesh_ldynak_quad.argtypes = [C.c_char_p, C.POINTER(fp), ip, C.POINTER(ip), ip]
    L.mfree_free.argtypes = [P]
    L.mfree_set_kernel_timing.argtypes = [P, I]
    L.mfree_get_kernel_times.argtypes = [P, C.POINTER(C.c_double), ip]
    L.mfree_probe_fp32_peak.argtypes = [C.POINTER(C.c_double)]
    L.mfree_timer_start.argtypes = [P]
    L.mfree_timer_stop.argtypes = [P, C.POINTER(C.c_double)]
    L.mfree_set_device.argtypes = [I]
    L.mfree_cell_list_static.argtypes = [P, I, fp, F, I, I, I, P, P, P]
    S, LL = C.c_size_t, C.c_longlong
    L.mfree_batch_create.argtypes = [S, P, C.POINTER(P)]
    L.mfree_batch_destroy.argtypes = [P]
    L.mfree_batch_admit.argtypes = [P, P, LL, ip]
    L.mfree_batch_step.argtypes = [P, I, I, I]
    L.mfree_batch_query.argtypes = [P, I, C.POINTER(LL), C.POINTER(LL), ip]
    L.mfree_batch_context.argtypes = [P, I, C.POINTER(P)]
    L.mfree_batch_retire.argtypes = [P, I, C.POINTER(P)]
    L.mfree_batch_info.argtypes = [P, ip, ip, C.POINTER(S), C.POINTER(S)]
    L.mfree_batch_set_tiling.argtypes = [P, I, I]
    L.mfree_batch_get_tiling.argtypes = [P, ip, ip]
    L.mfree_batch_autotune.argtypes = [P, I, ip, ip, C.POINTER(C.c_double)]
    L.mfree_batch_sync.argtypes = [P]
    L.mfree_batch_timer_start.argtypes = [P]
    L.mfree_batch_timer_stop.argtypes = [P, C.POINTER(C.c_double)]
    L.mfree_device_bytes.argtypes = [P, C.POINTER(S)]
    L.mfree_scene_bytes.argtypes = [I, LL]
    L.mfree_scene_bytes.restype = S
    for name in ("mfree_write_vtk", "mfree_write_vtk_tools", "mfree_write_vtk_blanking", "mfree_append_force_log"):
        getattr(L, name).argtypes = [P, C.c_char_p]
    L.mfree_output_wait.argtypes = [P]
    L.mfree_export_state.argtypes = [P, P, C.POINTER(S)]
    L.mfree_inject_fault.argtypes = [P, I]
    L.mfree_import_state.argtypes = [P, S, P, C.POINTER(P)]
    _lib = L
    return L


def _check(st: int):
    if st != 0:
        raise MfreeError(st, lib().mfree_last_error().decode())


def _f32(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(C.POINTER(C.c_float))


def _mk(cls, d):
    return cls(**{k: d[k] for k, _ in cls._fields_})


def set_device(device: int):
    """Select the CUDA device of the contexts created afterwards (one process per GPU)."""
    _check(lib().mfree_set_device(int(device)))


def fp32_peak_tflops() -> float:
    """Measured sustained FP32 FMA throughput of the current device (TFLOP/s)."""
    v = C.c_double()
    _check(lib().mfree_probe_fp32_peak(C.byref(v)))
    return v.value


def read_mesh(path: str, hexahedra: bool = False):
    """Read a MeshLab .json or LS-DYNA .k tool mesh (tetrahedral solids, or
    hexahedral ones with hexahedra=True): (verts (nv,3) float32, tris (nt,3) int32)."""
    L = lib()
    vp = C.POINTER(C.c_float)()
    tp = C.POINTER(C.c_int)()
    nv = C.c_int()
    nt = C.c_int()
    if path.endswith(".json"):
        fn = L.mfree_read_mesh_json
    else:
        fn = L.mfree_read_mesh_ldynak_quad if hexahedra else L.mfree_read_mesh_ldynak
    st = fn(path.encode(), C.byref(vp), C.byref(nv), C.byref(tp), C.byref(nt))
    if st != 0:
        raise MfreeError(st, f"could not read mesh {path}")
    try:
        v = np.ctypeslib.as_array(vp, shape=(nv.value * 3,)).copy().reshape(-1, 3)
        t = np.ctypeslib.as_array(tp, shape=(nt.value * 3,)).copy().reshape(-1, 3)
    finally:
        L.mfree_free(vp)
        L.mfree_free(tp)
    return v, t


class Simulation:
    """One cutting scene on the GPU: particle_gpu + leap_frog + grid + blanking + tools."""

    def __init__(self, pos4, vel4, rho, h, T=None, fixed=None, tool_p=None, stream: Optional[int] = None):
        L = lib()
        self.L = L
        n = int(np.asarray(pos4).shape[0])
        keep = []

        def arg(a):
            if a is None:
                return None
            a, p = _f32(a)
            keep.append(a)
            return p

        h_ = C.c_void_p()
        _check(L.mfree_create(n, arg(pos4), arg(vel4), arg(rho), arg(T), arg(h), arg(fixed), arg(tool_p),
                              C.c_void_p(stream) if stream else None, C.byref(h_)))
        self.h = h_
        self.n_init = n
        self.num_tools = 0

    # -- the reference's setup calls --
    def set_physics(self, **kw):
        self._phys = _mk(Phys, kw)
        _check(self.L.mfree_set_physics(self.h, C.byref(self._phys)))

    def set_correctors(self, **kw):
        self._corr = _mk(Corr, kw)
        _check(self.L.mfree_set_correctors(self.h, C.byref(self._corr)))

    def set_johnson_cook(self, **kw):
        self._joco = _mk(Joco, kw)
        _check(self.L.mfree_set_johnson_cook(self.h, C.byref(self._joco)))

    def set_thermal_workpiece(self, **kw):
        self._twp = _mk(Trml, kw)
        _check(self.L.mfree_set_thermal_workpiece(self.h, C.byref(self._twp)))

    def set_thermal_tool(self, **kw):
        self._ttool = _mk(Trml, kw)
        _check(self.L.mfree_set_thermal_tool(self.h, C.byref(self._ttool)))

    def set_options(self, **kw):
        o = Options(cspm=0, conduction=COND_BROOKSHAW, precision=0, max_secant_iter=100, lanes_per_particle=0,
                    diagnostics=0, friction_tool_vel=0, tile_depth=0, full_stencil=0)
        for k, v in kw.items():
            setattr(o, k, int(v))
        self._opt = o
        _check(self.L.mfree_set_options(self.h, C.byref(o)))

    def options(self) -> dict:
        o = Options()
        _check(self.L.mfree_get_options(self.h, C.byref(o)))
        return {k: getattr(o, k) for k, _ in Options._fields_}

    def set_grid(self, bbmin, bbmax, h: float):
        lo, plo = _f32(bbmin)
        hi, phi = _f32(bbmax)
        _check(self.L.mfree_set_grid(self.h, plo, phi, float(h)))

    def set_grid_adaptive(self, max_cell: int):
        """The unlocked grid (grid_gpu_green(max_cell, N)): box and cell edge from the particles every step."""
        _check(self.L.mfree_set_grid_adaptive(self.h, int(max_cell)))

    def set_grid_velocity(self, vel):
        v, p = _f32(vel)
        _check(self.L.mfree_set_grid_velocity(self.h, p))

    def set_blanking(self, bbmin, bbmax, max_vel: float, bbvel=None):
        lo, plo = _f32(bbmin)
        hi, phi = _f32(bbmax)
        vv = None
        if bbvel is not None:
            vv_a, vv = _f32(bbvel)
        _check(self.L.mfree_set_blanking(self.h, plo, phi, vv, float(max_vel)))

    def set_time(self, dt: float, t: float):
        _check(self.L.mfree_set_time(self.h, float(dt), float(t)))

    def time(self):
        dt = C.c_float()
        t = C.c_float()
        _check(self.L.mfree_get_time(self.h, C.byref(dt), C.byref(t)))
        return dt.value, t.value

    def add_tool(self, verts, tris, vel, contact_alpha: float = 0.1, mu: float = 0.0,
                 algorithm: int = CONTACT_HASHED) -> int:
        v, pv = _f32(np.asarray(verts).reshape(-1))
        t = np.ascontiguousarray(np.asarray(tris, np.int32).reshape(-1))
        ve, pve = _f32(vel)
        k = C.c_int()
        _check(self.L.mfree_add_tool(self.h, pv, len(v) // 3, t.ctypes.data_as(C.POINTER(C.c_int)), len(t) // 3,
                                     pve, float(contact_alpha), float(mu), int(algorithm), C.byref(k)))
        self.num_tools += 1
        return k.value

    def tool_info(self, k: int = 0) -> dict:
        nt, nb = C.c_int(), C.c_int()
        n3 = (C.c_int * 3)()
        lo = (C.c_float * 3)()
        hi = (C.c_float * 3)()
        dx = C.c_float()
        _check(self.L.mfree_get_tool_info(self.h, k, C.byref(nt), C.byref(nb), n3, lo, hi, C.byref(dx)))
        return dict(num_tris=nt.value, num_boxed=nb.value, n3=tuple(n3), bbmin=tuple(lo), bbmax=tuple(hi),
                    dx=dx.value)

    def tool_normals(self, k: int = 0) -> np.ndarray:
        nt = self.tool_info(k)["num_tris"]
        out = np.zeros(nt * 21, np.float32)
        _check(self.L.mfree_get_tool_normals(self.h, k, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out.reshape(nt, 7, 3)

    def tool_cells(self, k: int = 0):
        info = self.tool_info(k)
        nc = info["n3"][0] * info["n3"][1] * info["n3"][2]
        cells = np.zeros(nc + 1, np.int32)
        src = np.zeros(max(1, info["num_boxed"]), np.int32)
        ip = C.POINTER(C.c_int)
        _check(self.L.mfree_get_tool_cells(self.h, k, cells.ctypes.data_as(ip), src.ctypes.data_as(ip)))
        return cells, src[: info["num_boxed"]]

    def tool_forces(self) -> np.ndarray:
        out = np.zeros(3 * max(1, self.num_tools), np.float32)
        _check(self.L.mfree_get_tool_forces(self.h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out.reshape(-1, 3)[: self.num_tools]

    # -- stepping --
    def step(self, record_forces: bool = False):
        _check(self.L.mfree_step(self.h, int(record_forces)))

    def advance(self, nsteps: int, record_every: int = 0, use_graph: bool = True):
        _check(self.L.mfree_advance(self.h, int(nsteps), int(record_every), int(use_graph)))

    def set_kernel_timing(self, on: bool = True):
        _check(self.L.mfree_set_kernel_timing(self.h, int(on)))

    def kernel_times(self) -> dict:
        """{kernel: (total ms, launches)} of the eager steps since the last call."""
        ms = (C.c_double * len(KERNELS))()
        n = (C.c_int * len(KERNELS))()
        _check(self.L.mfree_get_kernel_times(self.h, ms, n))
        return {k: (ms[i], n[i]) for i, k in enumerate(KERNELS)}

    def timer_start(self):
        _check(self.L.mfree_timer_start(self.h))

    def timer_stop(self) -> float:
        """Device milliseconds since timer_start (CUDA events on the context's stream)."""
        ms = C.c_double()
        _check(self.L.mfree_timer_stop(self.h, C.byref(ms)))
        return ms.value

    def sync(self):
        _check(self.L.mfree_sync(self.h))

    # -- state --
    def counts(self):
        n = C.c_int()
        ni = C.c_int()
        _check(self.L.mfree_get_counts(self.h, C.byref(n), C.byref(ni)))
        return n.value, ni.value

    def inject_fault(self, kind: int):
        """Failure injection for tests: 1 makes the pair kernel's staging waits run out, 0 clears."""
        _check(self.L.mfree_inject_fault(self.h, int(kind)))

    def counters(self) -> dict:
        c = Counters()
        _check(self.L.mfree_get_counters(self.h, C.byref(c)))
        return {k: getattr(c, k) for k, _ in Counters._fields_}

    def get(self, name: str, out: Optional[np.ndarray] = None) -> np.ndarray:
        """A whole field; ``out`` (C-contiguous, n_init x width entries of the
        field's dtype) is filled instead of a new array -- page-locked memory
        there lets the device write the field directly."""
        f = FIELD_ID[name]
        w = self.L.mfree_field_width(f)
        dt = np.int32 if name in INT_FIELDS else np.float32
        if out is None:
            out = np.zeros(self.n_init * w, dt)
        elif out.dtype != dt or out.size != self.n_init * w or not out.flags["C_CONTIGUOUS"]:
            raise ValueError(f"get({name!r}): out must be a C-contiguous {np.dtype(dt).name} array of "
                             f"{self.n_init * w} entries")
        _check(self.L.mfree_get_field(self.h, f, out.ctypes.data_as(C.c_void_p)))
        return out.reshape(self.n_init, w) if w > 1 else out.reshape(-1)

    def get_array(self, name: str, out: Optional[np.ndarray] = None) -> np.ndarray:
        """One of the library's own float4 arrays (ARRAYS), n_init x 4."""
        if out is None:
            out = np.empty((self.n_init, 4), np.float32)
        elif out.dtype != np.float32 or out.size != 4 * self.n_init or not out.flags["C_CONTIGUOUS"]:
            raise ValueError(f"get_array({name!r}): out must be a C-contiguous float32 array of {4 * self.n_init}")
        _check(self.L.mfree_get_array(self.h, ARRAYS.index(name), out.ctypes.data_as(C.POINTER(C.c_float))))
        return out.reshape(self.n_init, 4)

    def set_array(self, name: str, values):
        a = np.ascontiguousarray(values, dtype=np.float32).reshape(-1)
        if a.size != 4 * self.n_init:
            raise ValueError(f"set_array({name!r}): {4 * self.n_init} floats expected")
        _check(self.L.mfree_set_array(self.h, ARRAYS.index(name), a.ctypes.data_as(C.POINTER(C.c_float))))

    def energies(self) -> dict:
        """FP64 device reductions: kinetic, deviatoric and volumetric elastic, thermal energy and the CFL bound."""
        out = (C.c_double * 5)()
        _check(self.L.mfree_get_energies(self.h, out))
        return dict(kinetic=out[0], elastic_deviatoric=out[1], elastic_volumetric=out[2], thermal=out[3],
                    cfl_dt=out[4])

    def array_device_ptr(self, name: str) -> int:
        p = C.c_void_p()
        _check(self.L.mfree_array_device_ptr(self.h, ARRAYS.index(name), C.byref(p)))
        return int(p.value or 0)

    def get64(self, name: str) -> np.ndarray:
        f = FIELD_ID[name]
        w = self.L.mfree_field_width(f)
        out = np.zeros(self.n_init * w, np.float64)
        _check(self.L.mfree_get_field_f64(self.h, f, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out.reshape(self.n_init, w) if w > 1 else out

    def set(self, name: str, values):
        a = np.ascontiguousarray(values, dtype=np.float32).reshape(-1)
        _check(self.L.mfree_set_field(self.h, FIELD_ID[name], a.ctypes.data_as(C.c_void_p)))

    def grid(self):
        nx, ny, nz = C.c_long(), C.c_long(), C.c_long()
        lo = (C.c_float * 3)()
        dx = C.c_float()
        _check(self.L.mfree_get_grid(self.h, C.byref(nx), C.byref(ny), C.byref(nz), lo, C.byref(dx)))
        return (nx.value, ny.value, nz.value), tuple(lo), dx.value

    def cells(self):
        (nx, ny, nz), _, _ = self.grid()
        cs = np.zeros(nx * ny * nz, np.int32)
        ce = np.zeros(nx * ny * nz, np.int32)
        ip = C.POINTER(C.c_int)
        _check(self.L.mfree_get_cells(self.h, cs.ctypes.data_as(ip), ce.ctypes.data_as(ip)))
        return cs, ce

    # -- checkpoint and resume
    def export_state(self) -> bytes:
        """The context (configuration, tools, clock, particle state) as one binary record."""
        n = C.c_size_t()
        _check(self.L.mfree_export_state(self.h, None, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        _check(self.L.mfree_export_state(self.h, buf, C.byref(n)))
        return buf.raw[: n.value]

    @classmethod
    def import_state(cls, record: bytes, stream: Optional[int] = None) -> "Simulation":
        """A new context from a record of export_state; it steps on exactly as the exported one."""
        import struct
        L = lib()
        h = C.c_void_p()
        buf = C.create_string_buffer(record, len(record))
        _check(L.mfree_import_state(buf, len(record), C.c_void_p(stream) if stream else None, C.byref(h)))
        sim = cls.__new__(cls)
        sim.L = L
        sim.h = h
        sim.n_init, sim.num_tools = struct.unpack_from("<II", record, 12)
        return sim

    # -- output in the reference's formats (results/vtk_out_%06d.vtk etc.)
    def write_vtk(self, path: str):
        """Particles as legacy VTK; written in the background (output_wait joins)."""
        _check(self.L.mfree_write_vtk(self.h, os.fsencode(path)))

    def output_wait(self):
        _check(self.L.mfree_output_wait(self.h))

    def write_vtk_tools(self, path: str):
        _check(self.L.mfree_write_vtk_tools(self.h, os.fsencode(path)))

    def write_vtk_blanking(self, path: str):
        _check(self.L.mfree_write_vtk_blanking(self.h, os.fsencode(path)))

    def append_force_log(self, path: str):
        _check(self.L.mfree_append_force_log(self.h, os.fsencode(path)))

    def device_bytes(self) -> int:
        """Device memory the context holds (state, scratch, tools)."""
        b = C.c_size_t()
        _check(self.L.mfree_device_bytes(self.h, C.byref(b)))
        return b.value

    def close(self):
        if getattr(self, "_batch", None) is not None:
            return  # a batch owns the context; Batch.retire / Batch.close release it
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.mfree_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- building from a scene description --
    @classmethod
    def from_scene(cls, scene, stream: Optional[int] = None, **option_overrides) -> "Simulation":
        """Set up a scene the way the reference's setup functions do."""
        s = cls(scene.pos, scene.vel, scene.rho, scene.h, T=scene.T, fixed=scene.fixed, tool_p=scene.tool_p,
                stream=stream)
        s.set_physics(**scene.phys)
        s.set_correctors(**scene.corr)
        if scene.joco:
            s.set_johnson_cook(**scene.joco)
        s.set_thermal_workpiece(**scene.trml_wp)
        s.set_thermal_tool(**scene.trml_tool)
        opts = dict(scene.options)
        opts.update(option_overrides)
        s.set_options(**opts)
        if scene.grid_max_cell > 0:
            s.set_grid_adaptive(scene.grid_max_cell)
        else:
            s.set_grid(scene.grid_bbmin, scene.grid_bbmax, scene.grid_h)
        s.set_blanking(scene.blank_bbmin, scene.blank_bbmax, scene.blank_vmax)
        for t in scene.tools:
            s.add_tool(t.verts, t.tris, t.vel, t.contact_alpha, t.mu, t.algorithm)
        # main() skips the step at index 0 and then advances the clock once
        dt = np.float32(scene.dt)
        s.set_time(float(dt), float(np.float32(0) + dt))
        return s


def scene_bytes(n: int, num_cell: int) -> int:
    """Device bytes mfree_create + mfree_set_grid take for n particles and num_cell cells (tools excluded)."""
    return int(lib().mfree_scene_bytes(int(n), int(num_cell)))


class Batch:
    """Independent scenes stepped together, one launch per kernel (mfree_batch_*).

    ``admit`` hands a configured ``Simulation`` to the batch (field reads keep
    working on it); ``step`` advances every running scene; a scene admitted
    with ``steps`` stops after that many steps; ``retire`` removes it.
    """
    RUNNING, DONE, FREE = 0, 1, 2

    def __init__(self, hbm_budget: int = 0, stream: Optional[int] = None):
        self.L = lib()
        h = C.c_void_p()
        _check(self.L.mfree_batch_create(int(hbm_budget), C.c_void_p(stream) if stream else None, C.byref(h)))
        self.h = h
        self.sims = {}

    def admit(self, sim: Simulation, steps: int = 0) -> Optional[int]:
        """Slot of the admitted scene, or None when it does not fit the memory budget."""
        k = C.c_int()
        st = self.L.mfree_batch_admit(self.h, sim.h, int(steps), C.byref(k))
        if st == ERR_BUDGET:
            return None
        _check(st)
        sim._batch = self
        self.sims[k.value] = sim
        return k.value

    def step(self, nsteps: int = 1, record_every: int = 0, use_graph: bool = True):
        _check(self.L.mfree_batch_step(self.h, int(nsteps), int(record_every), int(use_graph)))

    def query(self, slot: int):
        """(steps done, steps requested, status): status 0 running, 1 done, 2 free, < 0 error."""
        d, t, s = C.c_longlong(), C.c_longlong(), C.c_int()
        _check(self.L.mfree_batch_query(self.h, int(slot), C.byref(d), C.byref(t), C.byref(s)))
        return d.value, t.value, s.value

    def retire(self, slot: int, keep: bool = False) -> Optional[Simulation]:
        """Remove a scene; keep=True returns its Simulation (owned by the caller again)."""
        sim = self.sims.pop(int(slot))
        out = C.c_void_p()
        _check(self.L.mfree_batch_retire(self.h, int(slot), C.byref(out) if keep else None))
        sim._batch = None
        if keep:
            return sim
        sim.h = C.c_void_p()
        return None

    def info(self) -> dict:
        n, r = C.c_int(), C.c_int()
        b, bud = C.c_size_t(), C.c_size_t()
        _check(self.L.mfree_batch_info(self.h, C.byref(n), C.byref(r), C.byref(b), C.byref(bud)))
        return dict(scenes=n.value, running=r.value, bytes=b.value, budget=bud.value)

    def set_tiling(self, lanes_per_particle: int = 0, tile_depth: int = 0):
        _check(self.L.mfree_batch_set_tiling(self.h, int(lanes_per_particle), int(tile_depth)))

    def tiling(self):
        a, b = C.c_int(), C.c_int()
        _check(self.L.mfree_batch_get_tiling(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def autotune(self, trial_steps: int = 3):
        """Time every tiling on copies of the running scenes; keep the fastest: (lanes, depth, ms/step)."""
        a, b, ms = C.c_int(), C.c_int(), C.c_double()
        _check(self.L.mfree_batch_autotune(self.h, int(trial_steps), C.byref(a), C.byref(b), C.byref(ms)))
        return a.value, b.value, ms.value

    def sync(self):
        _check(self.L.mfree_batch_sync(self.h))

    def timer_start(self):
        _check(self.L.mfree_batch_timer_start(self.h))

    def timer_stop(self) -> float:
        """Device milliseconds since timer_start (CUDA events on the batch's stream)."""
        ms = C.c_double()
        _check(self.L.mfree_batch_timer_stop(self.h, C.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.mfree_batch_destroy(self.h)
            for sim in self.sims.values():
                sim._batch = None
                sim.h = C.c_void_p()
            self.sims = {}
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
