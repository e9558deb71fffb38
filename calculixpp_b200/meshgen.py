"""Seeded synthetic box meshes for the hex/wedge solid families.

The reference has no mesh generator on this path (its decks come from .inp files);
these structured meshes stand in for the decks the benchmark configurations describe.
Node numbering follows a doubled lattice ordered x-fastest, then y, then z, so the
CSR matrix has a narrow bandwidth and neighbouring elements share cache lines.

Element node orders follow CalculiX / the reference:
  C3D8  : shape8h.f corner order (src/fem/element.cpp:160-175)
  C3D20 : corners then edge midsides 9-20 (src/fem/element.cpp:177-239)
  C3D6  : triangle base then top (src/fem/element.cpp:241-253)
  C3D15 : corners then midsides 1-2,2-3,3-1,4-5,5-6,6-4,1-4,2-5,3-6 (element.cpp:255-330)
Wedges come from splitting each hex cell along the xy face diagonal between its
corners 1 and 3 (0-based), giving two positively oriented prisms per cell.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

C3D4, C3D10, C3D8, C3D8R, C3D20, C3D20R, C3D6, C3D15 = 0, 1, 2, 3, 4, 5, 6, 7
NODES = {C3D4: 4, C3D10: 10, C3D8: 8, C3D8R: 8, C3D20: 20, C3D20R: 20, C3D6: 6, C3D15: 15}
NGP = {C3D4: 1, C3D10: 4, C3D8: 8, C3D8R: 1, C3D20: 27, C3D20R: 8, C3D6: 2, C3D15: 6}
TYPE_NAMES = {C3D4: "C3D4", C3D10: "C3D10", C3D8: "C3D8", C3D8R: "C3D8R", C3D20: "C3D20", C3D20R: "C3D20R", C3D6: "C3D6", C3D15: "C3D15"}
NAMES = {C3D8: "C3D8", C3D8R: "C3D8R", C3D20: "C3D20", C3D20R: "C3D20R",
         C3D6: "C3D6", C3D15: "C3D15"}
BY_NAME = {v: k for k, v in NAMES.items()}

# Hex corner offsets in C3D8 order, on the unit cell.
_HEX = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                 [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.int64)
# C3D20 edges (pairs of corner indices) for midside nodes 9-20.
_HEX_EDGES = np.array([[0, 1], [1, 2], [2, 3], [3, 0], [4, 5], [5, 6],
                       [6, 7], [7, 4], [0, 4], [1, 5], [2, 6], [3, 7]])
# Wedge splits of a hex cell (corner indices into _HEX): bottom triangle + top.
_WEDGES = np.array([[0, 1, 3, 4, 5, 7], [1, 2, 3, 5, 6, 7]])
_W15_EDGES = np.array([[0, 1], [1, 2], [2, 0], [3, 4], [4, 5], [5, 3],
                       [0, 3], [1, 4], [2, 5]])
# Kuhn split of a hex cell into 6 tetrahedra along the main diagonal (corner 0 to
# corner 6 of _HEX): one per axis permutation, corners ordered for a positive Jacobian.
# Conforming across cells (every face is cut along the diagonal through its lowest
# corner).
_TETS = np.array([[0, 1, 2, 6], [0, 2, 3, 6], [0, 3, 7, 6], [0, 7, 4, 6], [0, 4, 5, 6], [0, 5, 1, 6]])
_T10_EDGES = np.array([[0, 1], [1, 2], [2, 0], [0, 3], [1, 3], [2, 3]])


@dataclass
class Mesh:
    """Nodes (N,3) float64, connectivity (E,n) int32 (0-based), one element type."""

    coords: np.ndarray
    conn: np.ndarray
    etype: int
    shape: tuple = ()
    young: np.ndarray | None = None
    poisson: np.ndarray | None = None
    extra: dict = field(default_factory=dict)

    @property
    def n_nodes(self) -> int:
        return int(self.coords.shape[0])

    @property
    def n_elems(self) -> int:
        return int(self.conn.shape[0])


def _lattice_nodes(n2, mask_fn):
    """Compact index for doubled-lattice points (x fastest) selected by mask_fn."""
    nx2, ny2, nz2 = n2
    z, y, x = np.meshgrid(np.arange(nz2), np.arange(ny2), np.arange(nx2), indexing="ij")
    mask = mask_fn(x, y, z)
    index = np.full(mask.shape, -1, dtype=np.int64)
    index[mask] = np.arange(int(mask.sum()))
    pts = np.stack([x[mask], y[mask], z[mask]], axis=1)
    return index, pts


def box_mesh(etype: int, nx: int, ny: int, nz: int, lx=1.0, ly=1.0, lz=1.0,
             jitter=0.0, seed=0, straight_edges=False) -> Mesh:
    """Structured box [0,lx]x[0,ly]x[0,lz] of nx*ny*nz hex cells.

    Hex types give one element per cell, wedge types two. Interior nodes (not on
    the box faces) move by uniform(-jitter*h, +jitter*h) per axis, h the cell size
    on that axis, drawn from numpy's default_rng(seed). With straight_edges, quadratic
    elements keep straight edges: the jittered corner nodes define the geometry and
    every midside node sits at the midpoint of its edge, so each quadratic element is
    exactly as regular as the linear cell under it.
    """
    if etype not in NODES:
        raise ValueError(f"unsupported element type {etype}")
    quadratic = etype in (C3D20, C3D20R, C3D15, C3D10)
    nc = np.array([nx, ny, nz], dtype=np.int64)
    if quadratic:
        n2 = 2 * nc + 1
        if etype == C3D15:
            def mask(x, y, z):
                return (z % 2 == 0) | ((x % 2 == 0) & (y % 2 == 0))
        elif etype == C3D10:
            def mask(x, y, z):
                return np.ones_like(x, dtype=bool)
        else:
            def mask(x, y, z):
                return ((x % 2) + (y % 2) + (z % 2)) <= 1
        index, pts = _lattice_nodes(n2, mask)
        scale = np.array([lx, ly, lz]) / (2 * nc)
    else:
        n2 = nc + 1
        index, pts = _lattice_nodes(n2, lambda x, y, z: np.ones_like(x, dtype=bool))
        scale = np.array([lx, ly, lz]) / nc
    coords = pts.astype(np.float64) * scale

    # Cell origins, x fastest.
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    cell = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1)
    step = 2 if quadratic else 1
    corner_lat = cell[:, None, :] * step + _HEX[None, :, :] * step  # (C,8,3)

    def lat_index(p):
        return index[p[..., 2], p[..., 1], p[..., 0]]

    if etype in (C3D8, C3D8R):
        conn = lat_index(corner_lat)
    elif etype in (C3D20, C3D20R):
        mids = (corner_lat[:, _HEX_EDGES[:, 0]] + corner_lat[:, _HEX_EDGES[:, 1]]) // 2
        conn = np.concatenate([lat_index(corner_lat), lat_index(mids)], axis=1)
    elif etype in (C3D4, C3D10):
        tet = corner_lat[:, _TETS].reshape(-1, 4, 3)
        if etype == C3D4:
            conn = lat_index(tet)
        else:
            mids = (tet[:, _T10_EDGES[:, 0]] + tet[:, _T10_EDGES[:, 1]]) // 2
            conn = np.concatenate([lat_index(tet), lat_index(mids)], axis=1)
    else:
        w = corner_lat[:, _WEDGES]  # (C,2,6,3)
        w = w.reshape(-1, 6, 3)
        if etype == C3D6:
            conn = lat_index(w)
        else:
            mids = (w[:, _W15_EDGES[:, 0]] + w[:, _W15_EDGES[:, 1]]) // 2
            conn = np.concatenate([lat_index(w), lat_index(mids)], axis=1)
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    if np.any(conn < 0):
        raise AssertionError("lattice index miss while building connectivity")

    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        h = np.array([lx / nx, ly / ny, lz / nz])
        lo = np.zeros(3)
        hi = np.array([lx, ly, lz])
        eps = 1e-9 * hi
        interior = np.all((coords > lo + eps) & (coords < hi - eps), axis=1)
        d = rng.uniform(-1.0, 1.0, size=coords.shape) * (jitter * h)
        coords = coords + d * interior[:, None]
        if straight_edges and quadratic:
            if etype == C3D15:
                nc_, edges = 6, _W15_EDGES
            elif etype == C3D10:
                nc_, edges = 4, _T10_EDGES
            else:
                nc_, edges = 8, _HEX_EDGES
            for i, (a, b) in enumerate(edges):
                coords[conn[:, nc_ + i]] = 0.5 * (coords[conn[:, a]] + coords[conn[:, b]])
    return Mesh(coords=np.ascontiguousarray(coords), conn=conn, etype=etype,
                shape=(nx, ny, nz))


def face_nodes(mesh: Mesh, axis: int, value: float, tol=1e-9) -> np.ndarray:
    """Node indices on the plane coords[:, axis] == value."""
    return np.nonzero(np.abs(mesh.coords[:, axis] - value) <= tol * max(1.0, abs(value) + 1.0))[0]


def clamp_face_spc(mesh: Mesh, axis=0, value=0.0):
    """SPC arrays (node, comp, value) fixing all three components on one face."""
    nodes = face_nodes(mesh, axis, value)
    spc_node = np.repeat(nodes, 3).astype(np.int32)
    spc_comp = np.tile(np.arange(3), nodes.size).astype(np.int32)
    return spc_node, spc_comp, np.zeros(spc_node.size)


def dof_map(n_nodes: int, spc_node, spc_comp, spc_val):
    """Free-DOF numbering of an SPC-only model, restating constraint_transform.cpp:78-82:
    free DOFs are numbered in global order g = 3*node + comp."""
    ndof = 3 * n_nodes
    constrained = np.zeros(ndof, dtype=bool)
    prescribed = np.zeros(ndof)
    g = 3 * np.asarray(spc_node, dtype=np.int64) + np.asarray(spc_comp, dtype=np.int64)
    constrained[g] = True
    prescribed[g] = spc_val
    dof_eq = np.full(ndof, -1, dtype=np.int32)
    free = ~constrained
    dof_eq[free] = np.arange(int(free.sum()), dtype=np.int32)
    return dof_eq, prescribed, int(free.sum())


def cantilever_c3d8_config1(seed=0) -> dict:
    """Plain FP64 linear-static C3D8 cantilever: 20x4x4 hexes of a 100x10x10 box,
    interior nodes jittered by uniform +-0.1*h, E=210000, nu=0.3, face x=0 clamped,
    total load -1000 in z split evenly over the x=100 face nodes."""
    m = box_mesh(C3D8, 20, 4, 4, 100.0, 10.0, 10.0, jitter=0.1, seed=seed)
    m.young = np.full(m.n_elems, 210000.0)
    m.poisson = np.full(m.n_elems, 0.3)
    spc = clamp_face_spc(m, 0, 0.0)
    tip = face_nodes(m, 0, 100.0)
    f_ext = np.zeros(3 * m.n_nodes)
    f_ext[3 * tip + 2] = -1000.0 / tip.size
    return {"mesh": m, "spc": spc, "f_ext": f_ext, "tip": tip}


def lognormal_young(n, median=200000.0, sigma=0.3, seed=0):
    rng = np.random.default_rng(seed + 7919)
    return median * np.exp(sigma * rng.standard_normal(n))


def c3d20_block(n=64, seed=0) -> dict:
    """C3D20 full-integration block: n^3 quadratic hexes of a unit cube, node jitter
    uniform +-0.05*h, per-element E lognormal (median 200000, sigma 0.3), nu=0.3.
    For displacement checks: z=0 face clamped, unit total load in +x on z=1."""
    m = box_mesh(C3D20, n, n, n, 1.0, 1.0, 1.0, jitter=0.05, seed=seed)
    m.young = lognormal_young(m.n_elems, seed=seed)
    m.poisson = np.full(m.n_elems, 0.3)
    spc = clamp_face_spc(m, 2, 0.0)
    top = face_nodes(m, 2, 1.0)
    f_ext = np.zeros(3 * m.n_nodes)
    f_ext[3 * top + 0] = 1.0 / top.size
    return {"mesh": m, "spc": spc, "f_ext": f_ext}


J2_E, J2_NU, J2_SY, J2_H = 210000.0, 0.3, 250.0, 1000.0


def j2_table(h=J2_H, sy=J2_SY, ep_max=1.0):
    """*PLASTIC table of linear isotropic hardening: {0: sy, ep_max: sy + h*ep_max}. The
    reference extrapolates the table flat beyond its last point (plasticity.cpp:74-78),
    so ep_max is set far above any reachable equivalent plastic strain."""
    return (np.array([0.0, ep_max]), np.array([sy, sy + h * ep_max]))


def graded_uniaxial_field(coords, eps_max, p=3.0, nu=J2_NU):
    """Displacement of a bar under a graded uniaxial ramp: axial strain
    eps(x) = eps_max * x^p along the unit cube's x axis, lateral contraction -nu*eps(x)
    about the cross-section centre. With p = 3 and eps_max = 0.5 % the points with
    x > (sigma_y/(E*eps_max))^(1/3) ~ 0.62 yield, i.e. ~40 % of the Gauss points."""
    x, y, z = coords[:, 0], coords[:, 1], coords[:, 2]
    eps = eps_max * x ** p
    u = np.empty_like(coords)
    u[:, 0] = eps_max * x ** (p + 1) / (p + 1)
    u[:, 1] = -nu * eps * (y - 0.5)
    u[:, 2] = -nu * eps * (z - 0.5)
    return u.reshape(-1)


def c3d8_j2_block(n=128, seed=0) -> dict:
    """J2 Newton workload: n^3 C3D8 cube (unit edge), E=210000, nu=0.3, sigma_y=250,
    linear isotropic hardening H=1000. Constraints: u_x = 0 on x=0, u_y = u_z = 0 at the
    origin, u_z = 0 at (0,1,0); u_x on x=1 follows the ramp (filled in per increment by
    `j2_increment`)."""
    m = box_mesh(C3D8, n, n, n, 1.0, 1.0, 1.0, jitter=0.0, seed=seed)
    m.young = np.full(m.n_elems, J2_E)
    m.poisson = np.full(m.n_elems, J2_NU)
    x0 = face_nodes(m, 0, 0.0)
    x1 = face_nodes(m, 0, 1.0)
    origin = int(np.argmin(np.abs(m.coords).sum(1)))
    corner = int(np.argmin(np.abs(m.coords - np.array([0.0, 1.0, 0.0])).sum(1)))
    sn = np.concatenate([x0, x1, [origin, origin, corner]]).astype(np.int32)
    sc = np.concatenate([np.zeros(x0.size + x1.size, np.int32), np.array([1, 2, 2], np.int32)])
    return {"mesh": m, "spc_node": sn, "spc_comp": sc, "x1": x1, "table": j2_table()}


def j2_increment(cfg, k, n_inc=10, eps_final=0.005):
    """(u, spc) of increment k of the ramp: the graded field at eps_max = eps_final*k/n_inc
    and the matching prescribed values."""
    m = cfg["mesh"]
    u = graded_uniaxial_field(m.coords, eps_final * k / n_inc)
    sn, sc = cfg["spc_node"], cfg["spc_comp"]
    return u, (sn, sc, u[3 * sn.astype(np.int64) + sc])


BATCH_TYPES = (C3D8, C3D8R, C3D20R, C3D6, C3D15)


def batch_box(etype, n_elems, jitter=0.1, seed=0, E=210000.0, nu=0.3):
    """One model of the batched workload: a box of about n_elems elements of etype
    (wedges: two per hex cell), cells h = 1 per axis, node jitter +-jitter*h (corner nodes;
    quadratic midside nodes at their edge midpoints), z=0 clamped, unit total load in +x
    on the top face."""
    cells = max(1, int(round(n_elems / (2 if etype in (C3D6, C3D15) else 1))))
    nx = max(1, int(round(cells ** (1.0 / 3.0))))
    ny = nx
    nz = max(1, int(round(cells / (nx * ny))))
    m = box_mesh(etype, nx, ny, nz, float(nx), float(ny), float(nz), jitter=jitter, seed=seed, straight_edges=True)
    m.young = np.full(m.n_elems, float(E))
    m.poisson = np.full(m.n_elems, float(nu))
    spc = clamp_face_spc(m, 2, 0.0)
    top = face_nodes(m, 2, float(nz))
    return m, spc, top


def batched_workload(n_models=256, min_elems=1000, max_elems=200000, seed=0, types=BATCH_TYPES):
    """The batched mixed-element workload: n_models independent boxes with element counts
    log-uniform in [min_elems, max_elems], element type drawn from `types`, node jitter
    +-0.1 h, E ~ U[70000, 210000] and nu ~ U[0.25, 0.35] per model. Returns a list of
    (mesh, spc, top-face nodes, E, nu)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_models):
        etype = int(types[rng.integers(len(types))])
        ne = float(np.exp(rng.uniform(np.log(min_elems), np.log(max_elems))))
        E = float(rng.uniform(70000.0, 210000.0))
        nu = float(rng.uniform(0.25, 0.35))
        m, spc, top = batch_box(etype, ne, 0.1, seed * 100003 + k, E, nu)
        out.append((m, spc, top, E, nu))
    return out


def adjoint_cantilever(nx=96, ny=96, nz=48, seed=0, E0=210000.0, nu=0.3, load=-1000.0):
    """Adjoint-sensitivity workload: nx*ny*nz C3D8 cantilever of unit cells, per-element
    E = E0 * rho^3 with rho ~ U[0.1, 1] (seeded), x=0 face clamped, total load `load` in
    z spread evenly over the nodes of the x = nx face."""
    m = box_mesh(C3D8, nx, ny, nz, float(nx), float(ny), float(nz), jitter=0.0, seed=seed)
    rho = np.random.default_rng(seed).uniform(0.1, 1.0, m.n_elems)
    m.young = E0 * rho ** 3
    m.poisson = np.full(m.n_elems, nu)
    spc = clamp_face_spc(m, 0, 0.0)
    tip = face_nodes(m, 0, float(nx))
    return {"mesh": m, "spc": spc, "cloads": (tip, np.full(tip.size, 2), np.full(tip.size, load / tip.size)),
            "rho": rho}


def thermal_dof_map(n_nodes, tbc_node, tbc_val):
    """Scalar temperature DOF map (build_thermal_dof_map, src/fem/thermal.cpp:71-90):
    prescribed nodes get -1 and their value (last writer wins), the others are numbered
    in node order. Returns (t_dof_eq[N], t_prescribed[N], n_free)."""
    fixed = np.zeros(n_nodes, dtype=bool)
    pre = np.zeros(n_nodes)
    for node, val in zip(np.asarray(tbc_node, dtype=np.int64), np.asarray(tbc_val, dtype=np.float64)):
        fixed[node] = True
        pre[node] = val
    deq = np.full(n_nodes, -1, dtype=np.int32)
    deq[~fixed] = np.arange(int((~fixed).sum()), dtype=np.int32)
    return deq, pre, int((~fixed).sum())
