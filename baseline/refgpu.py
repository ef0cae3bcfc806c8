"""The comparator arm: the reference's own GPU step (iwf_mfree_gpu_3d,
leap_frog::step, src/leap_frog.cu:121-195) built for sm_100a by
``baseline/build_ref_gpu.sh`` into ``baseline/_ref/ref_step_<variant>``.

This module writes a ``scenes.Scene`` into the driver's scene file, runs the
driver (``baseline/ref_step_main.cu``) in a child process, and reads back its
timing line and, on request, the particle state after the last step.  The
reference's physics switches are compile-time, so a scene runs on the build of
its variant: ``brookshaw`` (no CSPM, Brookshaw conduction) or ``cspm_pse``.

It is a comparator, used by ``bench.py`` and the tests; the library never
imports it.
"""
from __future__ import annotations

import json
import os
import subprocess
import tempfile
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
VARIANTS = ("brookshaw", "cspm_pse")


def binary(variant: str) -> str:
    return os.path.join(REF_DIR, f"ref_step_{variant}")


def variant_of(scene) -> Optional[str]:
    """The build a scene needs, or None when no build of the reference matches
    its switches (conduction off, CSPM with Brookshaw, PSE without CSPM)."""
    cspm = int(scene.options.get("cspm", 0))
    cond = int(scene.options.get("conduction", 1))
    if cspm == 0 and cond == 1:
        return "brookshaw"
    if cspm == 1 and cond == 2:
        return "cspm_pse"
    return None


def available(variant: str) -> bool:
    return os.access(binary(variant), os.X_OK)


def build(reference_root: Optional[str] = None, variants=VARIANTS) -> bool:
    """Builds the variants from the reference's sources when they are present
    ($MFREE_REFERENCE_ROOT, else a ``reference`` directory beside the
    repository); returns whether every variant is available."""
    root = reference_root or os.environ.get("MFREE_REFERENCE_ROOT") or os.path.join(
        os.path.dirname(os.path.dirname(HERE)), "reference")
    if not os.path.exists(os.path.join(root, "src", "leap_frog.cu")):
        return all(available(v) for v in variants)
    deps = [os.path.join(HERE, f) for f in ("build_ref_gpu.sh", "ref_compat.h", "ref_step_main.cu")]
    deps.append(os.path.join(os.path.dirname(HERE), "oracle", "ref_include", "glm", "glm.hpp"))
    deps.append(os.path.join(os.path.dirname(HERE), "oracle", "ref_include", "ref_prelude.h"))
    newest = max(os.path.getmtime(d) for d in deps)
    stale = [v for v in variants if not available(v) or os.path.getmtime(binary(v)) < newest]
    if stale:
        subprocess.check_call(["sh", os.path.join(HERE, "build_ref_gpu.sh"), root, *stale])
    return True


def _f32(a) -> bytes:
    return np.ascontiguousarray(a, np.float32).tobytes()


def write_scene(scene, path: str):
    """The driver's scene file: header, constants, particle arrays, an
    optional initial stress (``scene.S0``, (n, 9) in the reference's
    column-major mat3x3 layout), tools (layout read by ref_step_main.cu)."""
    p, c, t = scene.phys, scene.corr, scene.trml_wp
    jc = scene.joco or {}
    tt = scene.trml_tool
    with open(path, "wb") as f:
        f.write(b"MFREESC1")
        f.write(np.array([scene.n, len(scene.tools), 1 if scene.joco else 0, int(scene.options.get("cspm", 0)),
                          int(scene.options.get("conduction", 1))], np.int32).tobytes())
        f.write(_f32([p["E"], p["nu"], p["rho0"], p["K"], p["G"], p["mass"]]))
        f.write(_f32([c["wdeltap"], c["stresseps"], c["xspheps"], c["alpha"], c["beta"], c["eta"]]))
        f.write(_f32([jc.get(k, 0.0) for k in ("A", "B", "C", "n", "m", "Tmelt", "Tref", "eps_dot_ref",
                                                "clamp_temp")]))
        f.write(_f32([t["cp"], t["tq"], t["k"], t["alpha"], t["T_init"], t["eta"]]))
        f.write(_f32([tt["cp"], tt["tq"], tt["k"], tt["alpha"], tt["T_init"], tt["eta"]]))
        f.write(_f32(scene.grid_bbmin) + _f32(scene.grid_bbmax) + _f32([scene.grid_h]))
        f.write(_f32(scene.blank_bbmin) + _f32(scene.blank_bbmax) + _f32([scene.blank_vmax, scene.dt]))
        for a in (scene.pos, scene.vel, scene.rho, scene.T, scene.h, scene.fixed, scene.tool_p):
            f.write(_f32(a))
        S0 = getattr(scene, "S0", None)
        f.write(np.array([0 if S0 is None else 1], np.int32).tobytes())
        if S0 is not None:
            f.write(_f32(np.asarray(S0, np.float32).reshape(scene.n, 9)))
        for tool in scene.tools:
            f.write(np.array([len(tool.verts), len(tool.tris), int(tool.algorithm)], np.int32).tobytes())
            f.write(_f32(tool.vel) + _f32([tool.contact_alpha, tool.mu]))
            f.write(_f32(tool.verts) + np.ascontiguousarray(tool.tris, np.int32).tobytes())


def read_state(path: str) -> dict:
    """The driver's state file, in the reference's per-field layout and sorted
    order; ``ID`` is each row's creation index."""
    raw = open(path, "rb").read()
    if raw[:8] != b"MFREERS1":
        raise ValueError("not a state file")
    n, active, nt = np.frombuffer(raw, np.int32, 3, 8)
    off = 20
    out = {"N": int(active)}

    def take(name, dtype, width):
        nonlocal off
        cnt = int(n) * width
        a = np.frombuffer(raw, dtype, cnt, off).copy()
        off += 4 * cnt
        out[name] = a.reshape(int(n), width) if width > 1 else a

    take("ID", np.int32, 1)
    for name, w in (("POS", 4), ("VEL", 4), ("S", 9), ("RHO", 1), ("T", 1), ("EPS_PL", 1), ("BLANKED", 1),
                    ("FC", 3), ("FT", 3), ("POS_T", 3), ("VEL_T", 3), ("S_T", 9), ("RHO_T", 1), ("T_T", 1),
                    ("R", 9)):
        take(name, np.float32, w)
    out["TOOL_FORCES"] = np.frombuffer(raw, np.float32, 3 * int(nt), off).reshape(int(nt), 3).copy()
    return out


def run(scene, warmup: int, steps: int, state: bool = False, timeout: float = 1800.0) -> dict:
    """Runs warmup + steps steps of the reference's step on the scene; returns
    the driver's timing record, with ``state`` (read_state) when asked.  The
    tool forces in the state are those of the last step (recorded there)."""
    variant = variant_of(scene)
    if variant is None:
        raise ValueError("no build of the reference has this scene's physics switches")
    exe = binary(variant)
    if not available(variant):
        raise FileNotFoundError(exe)
    with tempfile.TemporaryDirectory(prefix="mfree_ref_") as d:
        sp = os.path.join(d, "scene.bin")
        write_scene(scene, sp)
        cmd = [exe, sp, str(int(warmup)), str(int(steps))]
        if state:
            cmd.append(os.path.join(d, "state.bin"))
        r = subprocess.run(cmd, cwd=d, capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference step failed ({r.returncode}): {r.stdout[-2000:]}\n{r.stderr[-2000:]}")
        line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
        rec = json.loads(line)
        rec["variant"] = variant
        if state:
            rec["state"] = read_state(os.path.join(d, "state.bin"))
    return rec
