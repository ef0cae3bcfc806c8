"""Shared helpers of the parity tests: run the CUDA path and the oracle on the
same scene and compare fields particle by particle (matched by particle id)."""
from __future__ import annotations

import numpy as np

import oracle
from iwf_mfree_gpu_3d_b200 import api

FIELDS = ["POS", "VEL", "S", "EPS_PL", "EPS_PL_DOT", "T", "RHO", "POS_T", "VEL_T", "S_T", "RHO_T", "T_T", "FC",
          "FT"]


def by_id(ids: np.ndarray, arr: np.ndarray) -> np.ndarray:
    out = np.empty_like(arr)
    out[ids.astype(np.int64)] = arr
    return out


def gpu_state(sim: api.Simulation, names=FIELDS, f64: bool = False) -> dict:
    ids = sim.get("ID")
    out = {}
    for n in names:
        a = sim.get64(n) if (f64 and n in ("POS", "VEL")) else sim.get(n).astype(np.float64)
        out[n] = by_id(ids, a)
    out["BLANKED"] = by_id(ids, sim.get("BLANKED").astype(np.float64))
    return out


def oracle_state(orc: oracle.Oracle, names=FIELDS) -> dict:
    ids = orc.field("ID")
    out = {n: by_id(ids, orc.field(n)) for n in names}
    out["BLANKED"] = by_id(ids, orc.field("BLANKED"))
    return out


def rel_l2(a: np.ndarray, b: np.ndarray, mask=None) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if mask is not None:
        a = a[mask]
        b = b[mask]
    den = np.linalg.norm(b)
    num = np.linalg.norm(a - b)
    return float(num / den) if den > 0 else float(num)


def compare(g: dict, o: dict, scene, names=FIELDS) -> dict:
    """Per-field relative L2 error of the CUDA state against the oracle state;
    positions are compared as displacements, temperature as T - T0."""
    mask = (g["BLANKED"] == 0) & (o["BLANKED"] == 0)
    p0 = scene.pos[:, :3].astype(np.float64)
    T0 = scene.T.astype(np.float64)
    res = {}
    for n in names:
        a, b = g[n], o[n]
        if n == "POS":
            a = a[:, :3] - p0
            b = b[:, :3] - p0
        elif n == "VEL":
            a = a[:, :3]
            b = b[:, :3]
        elif n == "T":
            a = a - T0
            b = b - T0
        res[n] = rel_l2(a, b, mask)
    res["blank_mismatch"] = int(((g["BLANKED"] != 0) != (o["BLANKED"] != 0)).sum())
    return res


def unlocked_grid(pos4: np.ndarray, h: np.ndarray, n: int):
    """The unlocked grid of grid_base::update_geometry (grid_gpu_base.cu:185-233)
    in the reference's FP32 arithmetic: the box of the first n particles
    +-1e-6 (float minus a double literal, stored as float), the largest h as
    the cell edge, ceil(length / edge) cells per axis."""
    p = np.asarray(pos4, np.float32)[:n, :3]
    mn, mx = p.min(axis=0), p.max(axis=0)
    bbmin = (mn.astype(np.float64) - 1e-6).astype(np.float32)
    bbmax = (mx.astype(np.float64) + 1e-6).astype(np.float32)
    dx = np.float32(np.asarray(h, np.float32)[:n].max()) * np.float32(2.0) / np.float32(2.0)
    n3 = tuple(int(np.ceil(np.float32(bbmax[d] - bbmin[d]) / dx)) for d in range(3))
    return n3, bbmin, np.float32(dx)
