"""Cutting scenes in the reference's cm-g-us unit system.

The reference builds its scenes in C++ setup functions (for example
setup_single_grain_1tool, src/Benchmarks/benchmarks_single_grain.cu:674-876):
an x-major particle lattice with z = -k*dx, steel/titanium constants in
cm-g-us, a rigid triangulated tool, a locked cell grid and a blanking box of
the lattice and tool padded by 15*dx, dt = 0.5*CFL*h/(sqrt(v_tool) + c0).

This module builds the same kind of scene with seeded, deterministic inputs:

  * ``orthogonal_cutting(nx, ny, nz, ...)``: a steel block cut by a 12-triangle
    wedge (0 deg rake, 7 deg clearance) at the +x face -- the 8k and 1M
    workloads;
  * ``single_grain(...)``: a block cut by a truncated icosphere grain;
  * ``mixed_specs(count, seed, ...)`` / ``mixed_scene(spec)``: the uneven
    scenes of the batched and served workloads (sizes log-uniform, cutting
    speed, depth, rake and Johnson-Cook A, B, n drawn per scene).

The scene is plain numpy data; the CUDA path (``api.Simulation``) and the CPU
oracle consume the same arrays.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

# ---------------------------------------------------------------- seeding --

_U64 = np.uint64


def splitmix64(seed: int, n: int) -> np.ndarray:
    """n outputs of the SplitMix64 generator (Steele, Lea, Flood 2014)."""
    with np.errstate(over="ignore"):
        k = np.arange(1, n + 1, dtype=np.uint64)
        x = _U64(seed & 0xFFFFFFFFFFFFFFFF) + k * _U64(0x9E3779B97F4A7C15)
        z = x
        z = (z ^ (z >> _U64(30))) * _U64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> _U64(27))) * _U64(0x94D049BB133111EB)
        return z ^ (z >> _U64(31))


def uniform_pm1(seed: int, n: int) -> np.ndarray:
    """n doubles uniform in [-1, 1) from SplitMix64."""
    u = (splitmix64(seed, n) >> _U64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return 2.0 * u - 1.0


# ------------------------------------------------------------------ scene --

@dataclasses.dataclass
class Tool:
    verts: np.ndarray          # (nv, 3) float32
    tris: np.ndarray           # (nt, 3) int32, closed manifold
    vel: np.ndarray            # (3,) float32, cm/us
    contact_alpha: float = 0.1  # tool_3d_gpu.h:131-134 default
    mu: float = 0.35
    algorithm: int = 0         # 0 = spatial hashing (safe), 1 = exhaustive


@dataclasses.dataclass
class Scene:
    name: str
    pos: np.ndarray            # (n, 4) float32
    vel: np.ndarray            # (n, 4) float32
    rho: np.ndarray            # (n,) float32
    T: np.ndarray
    h: np.ndarray
    fixed: np.ndarray
    tool_p: np.ndarray
    phys: dict
    corr: dict
    joco: Optional[dict]
    trml_wp: dict
    trml_tool: dict
    options: dict
    grid_bbmin: np.ndarray
    grid_bbmax: np.ndarray
    grid_h: float
    blank_bbmin: np.ndarray
    blank_bbmax: np.ndarray
    blank_vmax: float
    dt: float
    tools: List[Tool]
    grid_max_cell: int = 0     # > 0: unlocked grid (box and cell edge from the particles every step)

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])


# steel in cm-g-us (E, K, G in Mbar; 1 Mbar = 1e11 Pa)
STEEL = dict(rho0=7.83, E=2.0, nu=0.29)
STEEL_JC = dict(A=7.92e-3, B=5.10e-3, C=0.014, n=0.26, m=1.03, Tmelt=1793.0, Tref=300.0,
                eps_dot_ref=1e-6, clamp_temp=1.0)


def kernel_value(r: float, h: float) -> float:
    """cubic_spline value W(r, h) (src/kernels.cuh:26-69), in double."""
    q = r / h
    fac = 1.0 / math.pi / h ** 3
    if q > 1.0:
        return 0.25 * (2.0 - q) ** 3 * fac
    return (1.0 - 1.5 * q * q * (1.0 - 0.5 * q)) * fac


def material(dx: float, hdx: float = 1.3, rho0=STEEL["rho0"], E=STEEL["E"], nu=STEEL["nu"],
             art_stress: float = 0.3):
    G = E / (2.0 * (1.0 + nu))
    K = 2.0 * G * (1.0 + nu) / (3.0 * (1.0 - 2.0 * nu))
    phys = dict(E=E, nu=nu, rho0=rho0, K=K, G=G, mass=dx ** 3 * rho0)
    corr = dict(wdeltap=kernel_value(dx, hdx * dx), stresseps=art_stress, xspheps=0.5,
                alpha=1.0, beta=1.0, eta=0.1)
    return phys, corr


def steel_thermal(rho0: float = STEEL["rho0"]):
    k = 50.0 * 1e-13        # W/(m K) -> cm-g-us
    cp = 477.0 * 1e-8       # J/(kg K) -> cm-g-us
    return dict(cp=cp, tq=0.9, k=k, alpha=k / (rho0 * cp), T_init=300.0, eta=0.9)


def time_step(h: float, v_tool: float, K: float, rho0: float, cfl: float = 0.3) -> float:
    """dt = 0.5 * CFL * h / (sqrt(v_tool) + c0) (benchmarks_single_grain.cu:849-851)."""
    c0 = math.sqrt(K / rho0)
    return float(np.float32(0.5 * cfl * h / (math.sqrt(v_tool) + c0)))


def wedge_tool(x_edge: float, z_edge: float, y0: float, y1: float, dx: float,
               rake_deg: float = 0.0, clearance_deg: float = 7.0,
               height: float = 10.0, length: float = 10.0):
    """Closed 12-triangle wedge (a hexahedron) cutting towards -x.

    Cross-section in x-z: cutting edge E=(x_edge, z_edge); the rake face rises
    from E to z_edge+height*dx, leaning back by the rake angle; the clearance face
    leaves E towards +x at the clearance angle; the tool is extruded over
    y0..y1."""
    H = height * dx
    L = length * dx
    zt = z_edge + H
    xr = x_edge + H * math.tan(math.radians(rake_deg))
    xc = x_edge + L
    zc = z_edge + L * math.tan(math.radians(clearance_deg))
    sec = [(x_edge, z_edge), (xr, zt), (xc + max(0.0, xr - x_edge), zt), (xc, zc)]
    v = []
    for y in (y0, y1):
        for (x, z) in sec:
            v.append((x, y, z))
    verts = np.array(v, dtype=np.float32)
    # quads of the hexahedron (vertices 0-3 at y0, 4-7 at y1)
    quads = [(0, 1, 2, 3), (4, 7, 6, 5), (0, 4, 5, 1), (1, 5, 6, 2), (2, 6, 7, 3), (3, 7, 4, 0)]
    tris = []
    for (a, b, c, d) in quads:
        tris.append((a, b, c))
        tris.append((a, c, d))
    return verts, np.array(tris, dtype=np.int32)


def lattice(nx: int, ny: int, nz: int, dx: float, seed: int = 0, jitter: float = 0.01):
    """x-major lattice (for i, for j, for k) with z = -k*dx and y centred, as
    benchmarks_single_grain.cu:720-737, plus a uniform +-jitter*dx per
    coordinate from SplitMix64."""
    ly = ny * dx
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    p = np.stack([i.ravel() * dx, j.ravel() * dx - ly / 2.0, -k.ravel() * dx], axis=1)
    n = p.shape[0]
    if jitter:
        p = p + jitter * dx * uniform_pm1(seed, 3 * n).reshape(n, 3)
    pos = np.zeros((n, 4), dtype=np.float32)
    pos[:, :3] = p.astype(np.float32)
    return pos


def orthogonal_cutting(nx: int = 40, ny: int = 20, nz: int = 10, dx: float = 1.0e-3,
                       v_tool: float = 1.0e-3, depth: float = 5.0, engage: float = 0.05,
                       seed: int = 0, cspm: bool = False, conduction: int = 1,
                       art_stress: float = 0.3, precision: int = 0, hdx: float = 1.3,
                       plastic: bool = True, algorithm: int = 0,
                       rake_deg: float = 0.0, jc_scale=(1.0, 1.0, 1.0),
                       name: Optional[str] = None) -> Scene:
    """Orthogonal cutting of a steel block by a rigid wedge.

    nx*ny*nz particles on a jittered lattice of spacing dx (cm); the wedge's
    cutting edge sits depth*dx below the top surface and overlaps the +x face
    by engage*dx (at 10 m/s the tool moves only ~4e-4 dx per step, so it has to
    start engaged); it moves towards -x at v_tool cm/us.  The bottom layer is
    fixed.  conduction: 0 none, 1 Brookshaw, 2 PSE."""
    h = hdx * dx
    pos = lattice(nx, ny, nz, dx, seed=seed)
    n = pos.shape[0]
    phys, corr = material(dx, hdx, art_stress=art_stress)
    joco = dict(STEEL_JC)
    joco["A"] *= jc_scale[0]
    joco["B"] *= jc_scale[1]
    joco["n"] *= jc_scale[2]
    twp = steel_thermal(phys["rho0"])
    ttool = dict(cp=0.0, tq=0.0, k=0.0, alpha=0.0, T_init=0.0, eta=0.0)
    lz = (nz - 1) * dx
    lx = (nx - 1) * dx
    ly = ny * dx
    fixed = (pos[:, 2] < -lz + dx / 2.0).astype(np.float32)
    verts, tris = wedge_tool(x_edge=lx - engage * dx, z_edge=-depth * dx,
                             y0=-ly / 2.0 - 2.0 * dx, y1=ly / 2.0 + 2.0 * dx, dx=dx,
                             rake_deg=rake_deg)
    tool = Tool(verts=verts, tris=tris, vel=np.array([-v_tool, 0.0, 0.0], np.float32),
                mu=0.35, contact_alpha=0.1, algorithm=algorithm)
    pad = 15.0 * dx
    lo = np.minimum(pos[:, :3].min(0), verts.min(0)) - pad
    hi = np.maximum(pos[:, :3].max(0), verts.max(0)) + pad
    dt = time_step(h, v_tool, phys["K"], phys["rho0"])
    options = dict(cspm=int(cspm), conduction=int(conduction), precision=int(precision),
                   max_secant_iter=100, lanes_per_particle=0, diagnostics=0, friction_tool_vel=0)
    return Scene(
        name=name or f"cut_{nx}x{ny}x{nz}",
        pos=pos,
        vel=np.zeros((n, 4), np.float32),
        rho=np.full(n, phys["rho0"], np.float32),
        T=np.full(n, twp["T_init"], np.float32),
        h=np.full(n, h, np.float32),
        fixed=fixed,
        tool_p=np.zeros(n, np.float32),
        phys=phys, corr=corr, joco=joco if plastic else None,
        trml_wp=twp, trml_tool=ttool, options=options,
        grid_bbmin=lo.astype(np.float32), grid_bbmax=hi.astype(np.float32), grid_h=float(np.float32(h)),
        blank_bbmin=lo.astype(np.float32), blank_bbmax=hi.astype(np.float32), blank_vmax=4.0,
        dt=dt, tools=[tool])


def two_tool_scene(nx: int = 40, ny: int = 20, nz: int = 10, dx: float = 1.0e-3, v_tool: float = 1.0e-3,
                   depths=(5.0, 3.0), engage=(0.05, 0.3), **kw) -> Scene:
    """Two rigid wedges cutting one block side by side, the way the
    reference's multi-grain setups step several tools in one contact pass
    (benchmarks_single_grain.cu:29-471; tools processed in order,
    leap_frog.cu:178-181): the first wedge covers the -y half of the block at
    depths[0]*dx, the second the +y half at depths[1]*dx, a dx apart.  Both
    move towards -x at v_tool; the grid and blanking box cover both."""
    sc = orthogonal_cutting(nx, ny, nz, dx, v_tool=v_tool, depth=depths[0], engage=engage[0], **kw)
    lx = (nx - 1) * dx
    ly = ny * dx
    halves = ((-ly / 2.0 - 2.0 * dx, -0.5 * dx), (0.5 * dx, ly / 2.0 + 2.0 * dx))
    algorithm = sc.tools[0].algorithm
    sc.tools = []
    for (y0, y1), depth, eng in zip(halves, depths, engage):
        verts, tris = wedge_tool(x_edge=lx - eng * dx, z_edge=-depth * dx, y0=y0, y1=y1, dx=dx)
        sc.tools.append(Tool(verts=verts, tris=tris, vel=np.array([-v_tool, 0.0, 0.0], np.float32),
                             mu=0.35, contact_alpha=0.1, algorithm=algorithm))
    pad = 15.0 * dx
    allv = np.concatenate([t.verts for t in sc.tools])
    lo = (np.minimum(sc.pos[:, :3].min(0), allv.min(0)) - pad).astype(np.float32)
    hi = (np.maximum(sc.pos[:, :3].max(0), allv.max(0)) + pad).astype(np.float32)
    sc.grid_bbmin, sc.grid_bbmax, sc.blank_bbmin, sc.blank_bbmax = lo, hi, lo.copy(), hi.copy()
    sc.name = f"two_tools_{nx}x{ny}x{nz}"
    return sc


def mesh_tool_scene(verts: np.ndarray, tris: np.ndarray, nx: int = 30, ny: int = 15, nz: int = 10,
                    dx: float = 1.0e-3, v_tool: float = 1.0e-3, depth: float = 3.0, engage: float = 0.05,
                    algorithm: int = 0, **kw) -> Scene:
    """A steel block cut by a tool read from a mesh file (api.read_mesh), placed
    the way the reference's single-grain setup places its LS-DYNA tool
    (benchmarks_single_grain.cu:689-707): lifted so that its lowest point lies
    depth*dx below the top surface, centred in y, and moved in x until its
    far side overlaps the block's -x face by engage*dx; it moves towards +x at
    v_tool.  Grid and blanking box cover block and tool, padded by 15*dx."""
    sc = orthogonal_cutting(nx, ny, nz, dx, v_tool=v_tool, **kw)
    v = np.asarray(verts, np.float64).copy()
    lo, hi = v.min(0), v.max(0)
    v[:, 2] += -lo[2] - depth * dx
    v[:, 1] += -lo[1] - (hi[1] - lo[1]) / 2.0
    v[:, 0] += -hi[0] + engage * dx
    sc.tools = [Tool(verts=v.astype(np.float32), tris=np.asarray(tris, np.int32),
                     vel=np.array([v_tool, 0.0, 0.0], np.float32), algorithm=algorithm)]
    pad = 15.0 * dx
    lo = (np.minimum(sc.pos[:, :3].min(0), v.min(0)) - pad).astype(np.float32)
    hi = (np.maximum(sc.pos[:, :3].max(0), v.max(0)) + pad).astype(np.float32)
    sc.grid_bbmin, sc.grid_bbmax, sc.blank_bbmin, sc.blank_bbmax = lo, hi, lo.copy(), hi.copy()
    sc.name = f"mesh_tool_{nx}x{ny}x{nz}"
    return sc


def small_scene(**kw) -> Scene:
    """40 x 20 x 10 = 8,000 particles, Brookshaw, no CSPM (the 8k workload)."""
    return orthogonal_cutting(40, 20, 10, **kw)


def million_scene(**kw) -> Scene:
    """200 x 100 x 50 = 1,000,000 particles, CSPM + artificial stress + PSE."""
    kw.setdefault("cspm", True)
    kw.setdefault("conduction", 2)
    return orthogonal_cutting(200, 100, 50, **kw)


# ------------------------------------------------------------ icosphere --

def icosphere(subdiv: int = 3, radius: float = 1.0):
    """Icosphere of 20 * 4**subdiv triangles (vertices on the sphere)."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    v = [np.array(p, float) / np.linalg.norm(p) for p in v]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
         (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[key] = len(v) - 1
            return cache[key]

        nf = []
        for (a, b, c) in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    return np.array(v) * radius, np.array(f, dtype=np.int32)


def truncated_grain(radius: float, rake_deg: float = -10.0, cut: float = 0.5):
    """Icosphere grain flattened by the rake plane: vertices beyond the plane
    are projected onto it, which keeps the 1,280 triangles and the mesh closed.
    The plane faces -x (the cutting direction), tilted by the rake angle."""
    v, f = icosphere(3, radius)
    a = math.radians(rake_deg)
    n = np.array([-math.cos(a), 0.0, math.sin(a)])   # outward normal of the rake face
    d = cut * radius
    s = v @ n - d
    v = v - np.maximum(s, 0.0)[:, None] * n[None, :]
    return v, f


def inside_mesh(points: np.ndarray, verts: np.ndarray, tris: np.ndarray, chunk: int = 2048) -> np.ndarray:
    """Points inside a closed triangle mesh: parity of the hits of a +z ray
    (Moller-Trumbore, the test the reference's contact uses)."""
    V = verts.astype(np.float64)
    v0, v1, v2 = V[tris[:, 0]], V[tris[:, 1]], V[tris[:, 2]]
    e1, e2 = v1 - v0, v2 - v0
    hv = np.stack([-e2[:, 1], e2[:, 0], np.zeros(len(e2))], 1)  # cross((0, 0, 1), e2)
    a = np.einsum("ij,ij->i", e1, hv)
    ok = np.abs(a) > 1e-12
    f = np.where(ok, 1.0 / np.where(ok, a, 1.0), 0.0)
    out = np.zeros(len(points), bool)
    P = points.astype(np.float64)
    for k in range(0, len(P), chunk):
        sv = P[k:k + chunk, None, :] - v0[None]
        u = f * np.einsum("mtj,tj->mt", sv, hv)
        q = np.cross(sv, e1[None])
        v = f * q[..., 2]
        t = f * np.einsum("tj,mtj->mt", e2, q)
        hit = ok & (u >= 0) & (u <= 1) & (v >= 0) & (u + v <= 1) & (t > 1e-12)
        out[k:k + chunk] = (hit.sum(1) % 2) == 1
    return out


def single_grain(nx: int = 400, ny: int = 160, nz: int = 64, dx: float = 1.0e-3, v_tool: float = 3.0e-3,
                 depth: float = 8.0, seed: int = 0, precision: int = 1, engage: float = 0.05,
                 tool_particles: bool = True, radius: float = 20.0) -> Scene:
    """Single-grain cutting: a 1,280-triangle truncated icosphere of radius
    radius*dx (20 by default) at 30 m/s, depth of cut 8*dx, Brookshaw
    conduction, compensated positions.  With
    tool_particles, the grain's volume outside the workpiece is sampled on the
    lattice spacing into tool particles (tool_p = 1) with diamond constants
    (k = 2200 W/mK, cp = 520 J/kgK, rho = 3500 kg/m^3, as the reference's
    single-grain setups, benchmarks_single_grain.cu:176,185-188), so heat flows
    into the tool through the particles the way the reference does it."""
    sc = orthogonal_cutting(nx, ny, nz, dx=dx, v_tool=v_tool, depth=depth, seed=seed,
                            precision=precision, name=f"grain_{nx}x{ny}x{nz}")
    R = radius * dx
    rake, cut = -10.0, 0.5
    v, f = truncated_grain(R, rake_deg=rake, cut=cut)
    lx = (nx - 1) * dx
    # lowest point depth*dx below the top surface; the flattened face, where it
    # crosses the top surface (its foremost point inside the block: the face
    # leans by the rake angle), overlaps the +x face by engage*dx, so the grain
    # is in contact from the first step
    v = v.copy()
    tz = -depth * dx - v[:, 2].min()
    a = math.radians(rake)
    nxp, nzp = -math.cos(a), math.sin(a)          # the face's outward normal (x, z); n . p = cut * R
    x_face = (cut * R - nzp * (-tz)) / nxp        # the face's x at local z = -tz (world z = 0)
    v[:, 0] += lx - engage * dx - x_face
    v[:, 2] += tz
    sc.tools = [Tool(verts=v.astype(np.float32), tris=f, vel=np.array([-v_tool, 0, 0], np.float32))]
    if tool_particles:
        lo, hi = v.min(0), v.max(0)
        axes = [np.arange(lo[d] + 0.5 * dx, hi[d], dx) for d in range(3)]
        g = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
        g = g[(g[:, 0] > lx + 0.5 * dx) & inside_mesh(g, v, f)]
        m = len(g)
        rho_d, cp_d, k_d = 3.5, 5.2e-6, 2.2e-10
        sc.pos = np.concatenate([sc.pos, np.concatenate([g, np.zeros((m, 1))], 1).astype(np.float32)])
        sc.vel = np.concatenate([sc.vel, np.zeros((m, 4), np.float32)])
        sc.rho = np.concatenate([sc.rho, np.full(m, rho_d, np.float32)])
        sc.T = np.concatenate([sc.T, np.full(m, sc.trml_wp["T_init"], np.float32)])
        sc.h = np.concatenate([sc.h, np.full(m, sc.h[0], np.float32)])
        sc.fixed = np.concatenate([sc.fixed, np.zeros(m, np.float32)])
        sc.tool_p = np.concatenate([sc.tool_p, np.ones(m, np.float32)])
        sc.trml_tool = dict(cp=cp_d, tq=0.0, k=k_d, alpha=k_d / (rho_d * cp_d), T_init=sc.trml_wp["T_init"], eta=0.0)
    pad = 15.0 * dx
    lo = np.minimum(sc.pos[:, :3].min(0), v.min(0)) - pad
    hi = np.maximum(sc.pos[:, :3].max(0), v.max(0)) + pad
    sc.grid_bbmin = sc.blank_bbmin = lo.astype(np.float32)
    sc.grid_bbmax = sc.blank_bbmax = hi.astype(np.float32)
    return sc


def five_grain_scene(nx: int = 24, ny: int = 44, nz: int = 10, dx: float = 1.0e-3, v_tool: float = 3.0e-3,
                     depth: float = 2.0, radius: float = 5.0, engage: float = 0.05, seed: int = 0,
                     precision: int = 0) -> Scene:
    """Five grains cutting one block, arranged as the reference's five-tool
    single-grain setup arranges its grain copies (benchmarks_single_grain.cu:
    29-471): a centre grain, two leading grains beside it at -+1.5 e in y, and
    two trailing grains e behind the leading row at -+0.5 e in y, e = 2
    radius (the grains do not overlap).  Each grain is the truncated icosphere
    of single_grain (radius*dx, -10 deg rake) at depth*dx below the top
    surface, all moving towards -x at v_tool: the leading row overlaps the
    block's +x face by engage*dx and is in contact from the first step, the
    trailing row reaches the block later.  Five tools in one contact pass, in
    list order."""
    sc = orthogonal_cutting(nx, ny, nz, dx=dx, v_tool=v_tool, depth=depth, seed=seed, precision=precision,
                            name=f"five_grains_{nx}x{ny}x{nz}")
    R = radius * dx
    e = 2.0 * R
    rake, cut = -10.0, 0.5
    v, f = truncated_grain(R, rake_deg=rake, cut=cut)
    lx = (nx - 1) * dx
    tz = -depth * dx - v[:, 2].min()
    a = math.radians(rake)
    nxp, nzp = -math.cos(a), math.sin(a)
    x_face = (cut * R - nzp * (-tz)) / nxp        # the face's x where it crosses the top surface
    base = v.copy()
    base[:, 0] += lx - engage * dx - x_face
    base[:, 2] += tz
    offsets = [(0.0, 0.0), (0.0, -1.5 * e), (0.0, 1.5 * e), (e, -0.5 * e), (e, 0.5 * e)]
    algorithm = sc.tools[0].algorithm
    sc.tools = []
    for ox, oy in offsets:
        g = base.copy()
        g[:, 0] += ox
        g[:, 1] += oy
        sc.tools.append(Tool(verts=g.astype(np.float32), tris=f, vel=np.array([-v_tool, 0.0, 0.0], np.float32),
                             algorithm=algorithm))
    pad = 15.0 * dx
    allv = np.concatenate([t.verts for t in sc.tools])
    lo = (np.minimum(sc.pos[:, :3].min(0), allv.min(0)) - pad).astype(np.float32)
    hi = (np.maximum(sc.pos[:, :3].max(0), allv.max(0)) + pad).astype(np.float32)
    sc.grid_bbmin, sc.grid_bbmax, sc.blank_bbmin, sc.blank_bbmax = lo, hi, lo.copy(), hi.copy()
    return sc


# ---------------------------------------------------- mixed-size workloads --

@dataclasses.dataclass
class MixedSpec:
    """One scene of a mixed workload: lattice nx = 4 nz, ny = 2 nz (n = 8 nz^3)."""
    nz: int
    v_tool: float       # cm/us
    depth: float        # in dx
    rake_deg: float
    jc_scale: tuple     # factors on Johnson-Cook A, B, n
    seed: int
    steps: int = 0      # steps a served request asks for

    @property
    def n(self) -> int:
        return 8 * self.nz ** 3


def mixed_specs(count: int, seed: int = 1, n_lo: int = 5000, n_hi: int = 200000, steps_lo: int = 0,
                steps_hi: int = 0) -> List[MixedSpec]:
    """Scenes with particle counts log-uniform in [n_lo, n_hi] (nz = round((n/8)^(1/3))),
    v ~ U[1e-4, 5e-3] cm/us (1-50 m/s), depth ~ U[2, 10] dx, rake ~ U[-20, 10] deg,
    Johnson-Cook A, B, n each x U[0.9, 1.1]; steps ~ U[steps_lo, steps_hi] when given."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for k in range(count):
        n = math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))
        nz = max(4, int(round((n / 8.0) ** (1.0 / 3.0))))
        v = float(rng.uniform(1.0e-4, 5.0e-3))
        depth = float(rng.uniform(2.0, 10.0))
        rake = float(rng.uniform(-20.0, 10.0))
        jc = tuple(float(x) for x in rng.uniform(0.9, 1.1, size=3))
        steps = int(rng.integers(steps_lo, steps_hi + 1)) if steps_hi > 0 else 0
        out.append(MixedSpec(nz=nz, v_tool=v, depth=depth, rake_deg=rake, jc_scale=jc, seed=seed * 100003 + k,
                             steps=steps))
    return out


def mixed_scene(spec: MixedSpec, precision: int = 1) -> Scene:
    """The cutting scene of a spec: the 8k scene's physics (Brookshaw, artificial
    stress, no CSPM) with compensated positions by default."""
    nz = spec.nz
    return orthogonal_cutting(4 * nz, 2 * nz, nz, v_tool=spec.v_tool, depth=min(spec.depth, nz - 2.0),
                              seed=spec.seed, rake_deg=spec.rake_deg, jc_scale=spec.jc_scale, precision=precision,
                              name=f"mixed_{4 * nz}x{2 * nz}x{nz}")
