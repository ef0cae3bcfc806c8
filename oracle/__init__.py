"""CPU oracle of the SPH cutting step -- TEST INFRASTRUCTURE.

Wraps ``oracle/liboracle.so`` (built from ``oracle/mfree_oracle.cpp``), a CPU
restatement of leap_frog::step of iwf_mfree_gpu_3d (src/leap_frog.cu:121-195)
in FP64 (and in the reference's FP32 semantics), and ``oracle/_ref/libref_kat.so``,
the reference's own kernel, eigen-solver and Johnson-Cook functions compiled
for the host from its sources (``oracle/build_ref.sh``).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this package; the product path never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_kat.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

# field ids and widths, same numbering as include/mfree.h
FIELDS = ["POS", "VEL", "VEL_BC", "H", "RHO", "P", "S", "R", "FC", "FT", "NRM", "FIXED", "BLANKED",
          "TOOL_PARTICLE", "EPS_PL", "EPS_PL_DOT", "T", "POS_T", "VEL_T", "RHO_T", "S_T", "T_T", "NUM_NBH",
          "IDX", "HASH", "ID", "POS_HALF"]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}
WIDTH = dict(POS=4, VEL=4, VEL_BC=4, S=9, R=9, FC=3, FT=3, NRM=3, POS_T=3, VEL_T=3, S_T=9, POS_HALF=4)


def build(force: bool = False) -> str:
    """Compile the oracle (g++ -O2 -fopenmp)."""
    src = os.path.join(HERE, "mfree_oracle.cpp")
    hdr = os.path.join(INCLUDE, "mfree.h")
    if (not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(src)
            and os.path.getmtime(LIB) >= os.path.getmtime(hdr)):
        return LIB
    cmd = ["g++", "-std=c++17", "-O2", "-fopenmp", "-fPIC", "-shared", "-I" + INCLUDE, src, "-o", LIB]
    subprocess.check_call(cmd)
    return LIB


def reference_root() -> str:
    """Where the reference's checkout is looked for: $MFREE_REFERENCE_ROOT, else
    a directory named ``reference`` beside this repository."""
    return os.environ.get("MFREE_REFERENCE_ROOT") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")


def build_ref(reference_root: str | None = None) -> str | None:
    """Compile the reference's functions for the host, when its sources exist."""
    reference_root = reference_root or globals()["reference_root"]()
    if not os.path.exists(os.path.join(reference_root, "src", "kernels.cuh")):
        return REF_LIB if os.path.exists(REF_LIB) else None
    subprocess.check_call(["sh", os.path.join(HERE, "build_ref.sh"), reference_root])
    return REF_LIB


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P, I, F, D, L_ = C.c_void_p, C.c_int, C.c_float, C.c_double, C.c_long
        fp = C.POINTER(C.c_float)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        lp = C.POINTER(C.c_long)
        L.orc_create.restype = P
        L.orc_create.argtypes = [I, I, fp, fp, fp, fp, fp, fp, fp]
        L.orc_destroy.argtypes = [P]
        L.orc_set_threads.argtypes = [I]
        L.orc_set_params.argtypes = [P, P, P, P, P, P, P]
        L.orc_set_grid.argtypes = [P, fp, fp, F]
        L.orc_set_grid_velocity.argtypes = [P, fp]
        L.orc_set_grid_adaptive.argtypes = [P, C.c_long]
        L.orc_set_blanking.argtypes = [P, fp, fp, fp, F]
        L.orc_set_time.argtypes = [P, D, D]
        L.orc_get_time.argtypes = [P]
        L.orc_get_time.restype = D
        L.orc_add_tool.argtypes = [P, fp, I, ip, I, fp, F, F, I]
        L.orc_tool_info.argtypes = [P, I, ip, ip, ip, fp, fp, fp]
        L.orc_tool_normals.argtypes = [P, I, dp]
        L.orc_tool_cells.argtypes = [P, I, ip, ip]
        L.orc_tool_forces.argtypes = [P, fp]
        L.orc_step.argtypes = [P, I]
        L.orc_counts.argtypes = [P, ip, ip]
        L.orc_secant_failures.argtypes = [P]
        L.orc_secant_failures.restype = L_
        L.orc_grid.argtypes = [P, lp, dp, dp]
        L.orc_cells.argtypes = [P, ip, ip]
        L.orc_get_field.argtypes = [P, I, dp]
        L.orc_set_field.argtypes = [P, I, dp]
        L.orc_last_error.argtypes = [P]
        L.orc_last_error.restype = C.c_char_p
        L.orc_hash_fp32.argtypes = [I, fp, fp, fp, F, L_, L_, L_, ip]
        L.orc_sort_cells.argtypes = [I, ip, I, L_, ip, ip, ip, ip]
        L.orc_neighbor_counts_fp32.argtypes = [I, fp, fp, ip, ip, ip, L_, L_, L_, ip]
        L.orc_cubic_spline.argtypes = [I, dp, dp, D, dp]
        L.orc_lapl_pse.argtypes = [I, dp, dp, D]
        L.orc_lapl_pse.restype = D
        L.orc_solve_eigen.argtypes = [I, dp, dp]
        L.orc_sigma_yield.argtypes = [I, dp, D, D, D]
        L.orc_sigma_yield.restype = D
        L.orc_solve_secant.argtypes = [I, dp, D, D, D, D, D, D, D, I, ip]
        L.orc_solve_secant.restype = D
        _lib = L
    return _lib


def ref_lib():
    """The reference's functions compiled for the host, or None when absent."""
    global _ref
    if _ref is None and os.path.exists(REF_LIB):
        R = C.CDLL(REF_LIB)
        fp = C.POINTER(C.c_float)
        D = C.c_double
        R.ref_cubic_spline.argtypes = [fp, fp, C.c_float, fp]
        R.ref_lapl_pse.argtypes = [fp, fp, C.c_float]
        R.ref_lapl_pse.restype = C.c_float
        R.ref_solve_eigen.argtypes = [fp, fp]
        R.ref_sigma_yield.argtypes = [fp, D, D, D]
        R.ref_sigma_yield.restype = D
        R.ref_solve_secant.argtypes = [fp, D, D, D, D, D, D, D, C.POINTER(C.c_int)]
        R.ref_solve_secant.restype = D
        _ref = R
    return _ref


def _f32(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(C.POINTER(C.c_float))


def _i32(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(C.POINTER(C.c_int))


def _f64(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


class _Phys(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("E", "nu", "rho0", "K", "G", "mass")]


class _Trml(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("cp", "tq", "k", "alpha", "T_init", "eta")]


class _Corr(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("wdeltap", "stresseps", "xspheps", "alpha", "beta", "eta")]


class _Joco(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("A", "B", "C", "n", "m", "Tmelt", "Tref", "eps_dot_ref", "clamp_temp")]


class _Opt(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("cspm", "conduction", "precision", "max_secant_iter",
                                       "lanes_per_particle", "diagnostics", "friction_tool_vel")]


def _mk(cls, d):
    return cls(**{k: d[k] for k, _ in cls._fields_})


class Oracle:
    """One scene stepped on the CPU (prec=64: FP64 restatement; prec=32: the
    reference's FP32 semantics)."""

    def __init__(self, scene, prec: int = 64, threads: int = 0):
        L = lib()
        self.L = L
        self.scene = scene
        if threads:
            L.orc_set_threads(threads)
        self._keep = []
        arrs = [scene.pos, scene.vel, scene.rho, scene.T, scene.h, scene.fixed, scene.tool_p]
        ptrs = []
        for a in arrs:
            a, p = _f32(a)
            self._keep.append(a)
            ptrs.append(p)
        self.h = L.orc_create(prec, scene.n, *ptrs)
        self.prec = prec
        self._phys = _mk(_Phys, scene.phys)
        self._corr = _mk(_Corr, scene.corr)
        self._joco = _mk(_Joco, scene.joco) if scene.joco else None
        self._twp = _mk(_Trml, scene.trml_wp)
        self._ttool = _mk(_Trml, scene.trml_tool)
        self._opt = _mk(_Opt, scene.options)
        L.orc_set_params(self.h, C.byref(self._phys), C.byref(self._corr),
                         C.byref(self._joco) if self._joco else None, C.byref(self._twp),
                         C.byref(self._ttool), C.byref(self._opt))
        lo, plo = _f32(scene.grid_bbmin)
        hi, phi = _f32(scene.grid_bbmax)
        if getattr(scene, "grid_max_cell", 0) > 0:
            L.orc_set_grid_adaptive(self.h, int(scene.grid_max_cell))
        else:
            L.orc_set_grid(self.h, plo, phi, scene.grid_h)
        blo, pblo = _f32(scene.blank_bbmin)
        bhi, pbhi = _f32(scene.blank_bbmax)
        L.orc_set_blanking(self.h, pblo, pbhi, None, scene.blank_vmax)
        for t in scene.tools:
            v, pv = _f32(t.verts.reshape(-1))
            tr, pt = _i32(t.tris.reshape(-1))
            vel, pvel = _f32(t.vel)
            k = L.orc_add_tool(self.h, pv, len(t.verts), pt, len(t.tris), pvel, t.contact_alpha, t.mu, t.algorithm)
            if k < 0:
                raise RuntimeError("oracle tool setup failed: " + L.orc_last_error(self.h).decode())
        # main() skips the step at index 0 and then advances the clock once
        dt32 = np.float32(scene.dt)
        L.orc_set_time(self.h, float(dt32), float(np.float32(0) + dt32))

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def set_time(self, dt: float, t: float):
        self.L.orc_set_time(self.h, dt, t)

    def step(self, record: bool = False):
        st = self.L.orc_step(self.h, int(record))
        if st != 0:
            raise RuntimeError(f"oracle step failed with status {st}")

    def run(self, n: int):
        for _ in range(n):
            self.step()

    def counts(self):
        n = C.c_int()
        ni = C.c_int()
        self.L.orc_counts(self.h, C.byref(n), C.byref(ni))
        return n.value, ni.value

    def field(self, name: str) -> np.ndarray:
        n = self.counts()[1]
        w = WIDTH.get(name, 1)
        out = np.zeros(n * w, np.float64)
        if self.L.orc_get_field(self.h, FIELD_ID[name], out.ctypes.data_as(C.POINTER(C.c_double))) != 0:
            raise KeyError(name)
        return out.reshape(n, w) if w > 1 else out

    def set_field(self, name: str, values: np.ndarray):
        v, p = _f64(np.asarray(values, np.float64).reshape(-1))
        if self.L.orc_set_field(self.h, FIELD_ID[name], p) != 0:
            raise KeyError(name)

    def grid(self):
        n3 = (C.c_long * 3)()
        lo = (C.c_double * 3)()
        dx = C.c_double()
        self.L.orc_grid(self.h, n3, lo, C.byref(dx))
        return tuple(n3), tuple(lo), dx.value

    def cells(self):
        (nx, ny, nz), _, _ = self.grid()
        nc = nx * ny * nz
        cs = np.zeros(nc, np.int32)
        ce = np.zeros(nc, np.int32)
        self.L.orc_cells(self.h, cs.ctypes.data_as(C.POINTER(C.c_int)), ce.ctypes.data_as(C.POINTER(C.c_int)))
        return cs, ce

    def tool_forces(self):
        out = np.zeros(3 * max(1, len(self.scene.tools)), np.float32)
        self.L.orc_tool_forces(self.h, out.ctypes.data_as(C.POINTER(C.c_float)))
        return out.reshape(-1, 3)

    def tool_info(self, k: int = 0):
        nt, nb = C.c_int(), C.c_int()
        n3 = (C.c_int * 3)()
        lo = (C.c_float * 3)()
        hi = (C.c_float * 3)()
        dx = C.c_float()
        self.L.orc_tool_info(self.h, k, C.byref(nt), C.byref(nb), n3, lo, hi, C.byref(dx))
        return dict(num_tris=nt.value, num_boxed=nb.value, n3=tuple(n3), bbmin=tuple(lo), bbmax=tuple(hi),
                    dx=dx.value)

    def tool_normals(self, k: int = 0):
        nt = self.tool_info(k)["num_tris"]
        out = np.zeros(nt * 21, np.float64)
        self.L.orc_tool_normals(self.h, k, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out.reshape(nt, 7, 3)

    def tool_cells(self, k: int = 0):
        info = self.tool_info(k)
        nc = info["n3"][0] * info["n3"][1] * info["n3"][2]
        cells = np.zeros(nc + 1, np.int32)
        src = np.zeros(info["num_boxed"], np.int32)
        self.L.orc_tool_cells(self.h, k, cells.ctypes.data_as(C.POINTER(C.c_int)),
                              src.ctypes.data_as(C.POINTER(C.c_int)))
        return cells, src

    def secant_failures(self) -> int:
        return int(self.L.orc_secant_failures(self.h))


# ---- FP32 integer pipeline of the reference (bit-exact checks) ----

def hash_fp32(pos4, blanked, bbmin, dx, n3):
    L = lib()
    p, pp = _f32(pos4)
    n = p.shape[0]
    b, pb = _f32(blanked if blanked is not None else np.zeros(n, np.float32))
    lo, plo = _f32(bbmin)
    out = np.zeros(n, np.int32)
    L.orc_hash_fp32(n, pp, pb, plo, float(dx), int(n3[0]), int(n3[1]), int(n3[2]),
                    out.ctypes.data_as(C.POINTER(C.c_int)))
    return out


def sort_cells(hash_, n_active, num_cell):
    L = lib()
    h, ph = _i32(hash_)
    n = h.shape[0]
    idx = np.zeros(n, np.int32)
    sh = np.zeros(n, np.int32)
    cs = np.zeros(num_cell, np.int32)
    ce = np.zeros(num_cell, np.int32)
    ip = C.POINTER(C.c_int)
    L.orc_sort_cells(n, ph, int(n_active), int(num_cell), idx.ctypes.data_as(ip), sh.ctypes.data_as(ip),
                     cs.ctypes.data_as(ip), ce.ctypes.data_as(ip))
    return idx, sh, cs, ce


def neighbor_counts_fp32(pos4, h, sorted_hash, cs, ce, n_active, n3):
    L = lib()
    p, pp = _f32(pos4)
    hh, ph = _f32(h)
    sh, psh = _i32(sorted_hash)
    a, pa = _i32(cs)
    b, pb = _i32(ce)
    out = np.zeros(int(n_active), np.int32)
    L.orc_neighbor_counts_fp32(int(n_active), pp, ph, psh, pa, pb, int(n3[0]), int(n3[1]), int(n3[2]),
                               out.ctypes.data_as(C.POINTER(C.c_int)))
    return out
