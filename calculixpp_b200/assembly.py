"""Python mirror of the reference's assembly interface, running on the B200 kernels.

Reference interface (include/calculixpp/fem/assembly.hpp, element.hpp):
    LinearSystem assemble_linear_static(const Model&)                    assembly.hpp:42
    MaterialPoints make_material_points(const Model&)                   assembly.hpp:93
    LinearSystem assemble_material_tangent(const Model&, u, mp, f_int)  assembly.hpp:105-108
    std::vector<Real> element_stiffness(type, coords, ElasticIso)       element.hpp:64-65
    ElementResponse element_tangent_force(type, coords, ue, material, state)
                                                                        element.hpp:160-164
Same names, same argument meaning, errors raised as exceptions carrying the reference's
messages. Differences: the stiffness comes back in canonical CSR (the reference's COO
triplets sorted by row then column), and arrays are torch tensors on the GPU. Every
call goes through the C ABI of libcxg.so (include/cxg.h); nothing here computes on the
CPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .meshgen import Mesh, NODES, NGP, dof_map

_vp = C.c_void_p


@dataclass
class Material:
    """ElasticIso + optional *PLASTIC table (core/material.hpp:81-115)."""

    E: float
    nu: float
    plastic: tuple | None = None  # (eqplastic[], yield[])
    hardening: int = 0            # 0 isotropic, 1 kinematic, 2 combined
    h_kin: float = 0.0


@dataclass
class Model:
    """The subset of cxpp::Model the assembly reads: mesh, per-element materials,
    single-point constraints (node, comp 0..2, value) and concentrated loads."""

    mesh: Mesh
    materials: list
    elem_mat: np.ndarray | None = None
    spc: tuple | None = None
    cloads: tuple | None = None

    def dof_map(self):
        sn, sc, sv = self.spc if self.spc is not None else (np.zeros(0, int), np.zeros(0, int), np.zeros(0))
        return dof_map(self.mesh.n_nodes, sn, sc, sv)

    def external_load_vector(self):
        """Full-magnitude CLOAD vector (src/fem/loads.cpp:575-585)."""
        f = np.zeros(3 * self.mesh.n_nodes)
        if self.cloads is not None:
            n, c, v = self.cloads
            np.add.at(f, 3 * np.asarray(n, dtype=np.int64) + np.asarray(c, dtype=np.int64), v)
        return f


@dataclass
class LinearSystem:
    """Reduced free/free system (assembly.hpp:18-38) with K_ff in CSR."""

    n_free: int
    row_ptr: torch.Tensor
    col_idx: torch.Tensor
    vals: torch.Tensor
    rhs: torch.Tensor
    dof_eq: np.ndarray
    prescribed: np.ndarray
    extra: dict = field(default_factory=dict)

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.vals.cpu().numpy(), self.col_idx.cpu().numpy(),
                              self.row_ptr.cpu().numpy()), shape=(self.n_free, self.n_free))


def _ptr(t):
    return None if t is None else _vp(t.data_ptr())


def _dev(a, dtype, device):
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=device)


def _stream():
    return _vp(torch.cuda.current_stream().cuda_stream)


def _c_material(m: Material, keep: list):
    cm = _lib.CxgMaterial()
    cm.E, cm.nu, cm.hardening, cm.h_kin = float(m.E), float(m.nu), int(m.hardening), float(m.h_kin)
    if m.plastic is None:
        cm.n_plastic, cm.eqplastic, cm.yield_ = 0, None, None
    else:
        ep = np.ascontiguousarray(m.plastic[0], dtype=np.float64)
        sy = np.ascontiguousarray(m.plastic[1], dtype=np.float64)
        keep += [ep, sy]
        cm.n_plastic = int(ep.size)
        cm.eqplastic, cm.yield_ = ep.ctypes.data, sy.ctypes.data
    return cm


class Plan:
    """A cxg_plan: mesh, DOF map and CSR pattern resident on one GPU."""

    def __init__(self, model: Model, precision: str = "fp64", device=None):
        self.lib = _lib.load()
        if not torch.cuda.is_available():
            raise _lib.CxgError(_lib.CXG_ERR_NO_GPU, "no CUDA device")
        self.device = torch.device(device or f"cuda:{torch.cuda.current_device()}")
        self.model = model
        self.precision = precision
        m = model.mesh
        dev = self.device
        dof_eq, prescribed, n_free = model.dof_map()
        self.dof_eq, self.prescribed, self.n_free = dof_eq, prescribed, n_free
        keep = []
        mats = (_lib.CxgMaterial * len(model.materials))(*[_c_material(x, keep) for x in model.materials])
        coords = _dev(m.coords, torch.float64, dev)
        conn = _dev(m.conn.reshape(-1), torch.int32, dev)
        young = _dev(m.young, torch.float64, dev) if m.young is not None else None
        poisson = _dev(m.poisson, torch.float64, dev) if m.poisson is not None else None
        elem_mat = _dev(model.elem_mat, torch.int32, dev) if model.elem_mat is not None else None
        d_dof = _dev(dof_eq, torch.int32, dev)
        d_pre = _dev(prescribed, torch.float64, dev)
        desc = _lib.CxgMeshDesc(m.n_nodes, m.n_elems, m.etype, _ptr(coords), _ptr(conn), _ptr(young),
                                _ptr(poisson), _ptr(elem_mat), len(model.materials),
                                C.cast(mats, _vp))
        dmap = _lib.CxgDofmapDesc(_ptr(d_dof), _ptr(d_pre), n_free)
        handle = _vp()
        with torch.cuda.device(dev):
            torch.cuda.synchronize()
            _lib.check(self.lib.cxg_plan_create(C.byref(desc), C.byref(dmap),
                                                _lib.MIXED if precision == "mixed" else _lib.FP64,
                                                C.byref(handle)))
        self.h = handle
        info = _lib.CxgPlanInfo()
        _lib.check(self.lib.cxg_plan_get_info(self.h, C.byref(info)))
        self.info = info
        self.nnz = int(info.nnz)
        self.n_gauss = int(info.n_gauss_points)
        rp, ci = _vp(), _vp()
        _lib.check(self.lib.cxg_plan_pattern_device(self.h, C.byref(rp), C.byref(ci)))
        self._pattern = None

    # -- lifetime ------------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.lib.cxg_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- pattern / precision -------------------------------------------------------
    def pattern(self):
        if self._pattern is None:
            rp = torch.empty(self.n_free + 1, dtype=torch.int64, device=self.device)
            ci = torch.empty(self.nnz, dtype=torch.int32, device=self.device)
            _lib.check(self.lib.cxg_plan_get_pattern(self.h, _ptr(rp), _ptr(ci)))
            self._pattern = (rp, ci)
        return self._pattern

    def set_precision(self, precision: str):
        _lib.check(self.lib.cxg_plan_set_precision(self.h, _lib.MIXED if precision == "mixed" else _lib.FP64))
        self.precision = precision

    def check(self):
        bad = C.c_int64()
        _lib.check(self.lib.cxg_plan_check(self.h, C.byref(bad)))

    def set_launch_config(self, tangent=False, tile=0, p1_blocks_per_sm=0, p2_warps=0):
        """Launch shape of the current precision's linear (or tangent) passes; tile 0 = 2x4,
        1 = 2x2, 2 = 4x4. Results do not depend on it."""
        _lib.check(self.lib.cxg_plan_set_launch_config(self.h, int(tangent), tile, p1_blocks_per_sm, p2_warps))

    def set_j2_fp32_return(self, enable=True):
        """Mixed precision, material-point assembly: the J2 return in FP32 (FP64 near the
        yield surface) instead of FP64 (cxg_plan_set_j2_fp32_return)."""
        _lib.check(self.lib.cxg_plan_set_j2_fp32_return(self.h, int(bool(enable))))

    def set_thermal_strain(self, node_temp=None, node_applied=None, elem_alpha=None, elem_tref=None):
        """Thermal-strain inputs (cxg_plan_set_thermal_strain; see `thermal_strain_inputs`):
        applied temperature per node, applied flags (None: all), expansion coefficient and
        reference temperature per element. node_temp None clears. The linear assembly then
        adds the thermal-strain load to the rhs and the recovery uses sigma = D (eps - eps_th)."""
        if node_temp is None:
            _lib.check(self.lib.cxg_plan_set_thermal_strain(self.h, None, None, None, None))
            return
        t = np.ascontiguousarray(node_temp, dtype=np.float64)
        ap = None if node_applied is None else np.ascontiguousarray(node_applied, dtype=np.uint8)
        al = np.ascontiguousarray(elem_alpha, dtype=np.float64)
        tr = np.ascontiguousarray(elem_tref, dtype=np.float64)
        if t.size != self.model.mesh.n_nodes or al.size != self.model.mesh.n_elems or tr.size != al.size:
            raise ValueError("node_temp[n_nodes], elem_alpha[n_elems] and elem_tref[n_elems] are required")
        ptr = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_plan_set_thermal_strain(self.h, ptr(t), ptr(ap), ptr(al), ptr(tr)))

    def thermal_strain_load(self):
        """thermal_strain_load_vector (src/fem/loads.cpp:515-560): f_th[3N] on the device."""
        out = torch.empty(3 * self.model.mesh.n_nodes, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_thermal_strain_load(self.h, _ptr(out), _stream()))
            self.check()
        return out

    def set_ring_bytes(self, nbytes: int):
        """Element-buffer budget of the windowed assembly (cxg_plan_set_ring_bytes):
        0 or < 0 = one window over the whole mesh, > 0 = windows whose buffers fit."""
        _lib.check(self.lib.cxg_plan_set_ring_bytes(self.h, int(nbytes)))

    def use_reference_pattern(self, enable=True):
        """Switch the linear assembly to the reference's own CSR pattern (entries whose
        every element contribution is exactly 0.0 in the reference's arithmetic dropped,
        cxg_plan_use_reference_pattern) or back to the topological one."""
        _lib.check(self.lib.cxg_plan_use_reference_pattern(self.h, int(bool(enable))))
        info = _lib.CxgPlanInfo()
        _lib.check(self.lib.cxg_plan_get_info(self.h, C.byref(info)))
        self.info = info
        self.nnz = int(info.nnz)
        self._pattern = None

    def windows(self, tangent=False):
        """(windows, elements held by the element buffers) of the last assembly of the
        current precision in this mode."""
        nw, ring = C.c_int32(), C.c_int64()
        _lib.check(self.lib.cxg_plan_get_windows(self.h, int(tangent), C.byref(nw), C.byref(ring)))
        return int(nw.value), int(ring.value)

    def tune(self, step, tangent=False, reps=3):
        """Time `step()` (one assembly through this plan) with CUDA events for every tile
        and element-pass grid shape of the current precision, then for the row gather's
        warps per block (8, 4, 2) at the kept element-pass shape, then for the
        element-buffer budget of the windowed assembly (one window, 40 % and 85 % of L2);
        keep the fastest and return it with its time in ms."""

        def timed(tile, bps, warps):
            try:
                self.set_launch_config(tangent, tile, bps, warps)
            except _lib.CxgError:
                return None
            step()
            torch.cuda.synchronize(self.device)
            t = []
            for _ in range(reps):
                s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s.record()
                step()
                e.record()
                e.synchronize()
                t.append(s.elapsed_time(e))
            return sorted(t)[len(t) // 2]

        # every launch shape is timed with one window first (a budget left by an earlier
        # tuning, e.g. of the other precision, would otherwise stand in for it)
        self.set_ring_bytes(0)
        best = None
        for tile in ((0, 1) if tangent else (0, 1, 2)):
            for bps in (0, 1, 2):
                ms = timed(tile, bps, 0)
                if ms is not None and (best is None or ms < best[0]):
                    best = (ms, tile, bps, 0)
        for warps in (4, 2):
            ms = timed(best[1], best[2], warps)
            if ms is not None and ms < best[0]:
                best = (ms, best[1], best[2], warps)
        # element-buffer budget: one window, or windows whose buffers take a share of L2
        # (results do not depend on it)
        l2 = torch.cuda.get_device_properties(self.device).L2_cache_size
        ring, ring_ms = 0, best[0]
        for budget in (int(0.4 * l2), int(0.85 * l2)):
            self.set_ring_bytes(budget)
            ms = timed(best[1], best[2], best[3])
            if ms is not None and ms < ring_ms:
                ring, ring_ms = budget, ms
        self.set_ring_bytes(ring)
        self.set_launch_config(tangent, best[1], best[2], best[3])
        return {"tile": {0: "2x4", 1: "2x2", 2: "4x4"}[best[1]], "p1_blocks_per_sm": best[2],
                "p2_warps": best[3] or 8, "ring_bytes": ring, "ms": ring_ms}

    # -- assembly --------------------------------------------------------------------
    def assemble_linear(self, f_ext=None, vals=None, rhs=None, check=True):
        dev = self.device
        vals = torch.empty(self.nnz, dtype=torch.float64, device=dev) if vals is None else vals
        rhs = torch.empty(self.n_free, dtype=torch.float64, device=dev) if rhs is None else rhs
        fe = None if f_ext is None else _dev(f_ext, torch.float64, dev)
        with torch.cuda.device(dev):
            _lib.check(self.lib.cxg_assemble_linear(self.h, _ptr(vals), _ptr(rhs), _ptr(fe), _stream()))
            if check:
                self.check()
        return vals, rhs

    def accumulate_linear(self, vals, rhs=None):
        """Add this plan's element contributions to vals (and rhs) in place; the element
        kernel alone, no zeroing and no load vector (cxg_assemble_linear_ex, CXG_ACCUMULATE)."""
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_assemble_linear_ex(self.h, _ptr(vals), _ptr(rhs), None, _lib.ACCUMULATE,
                                                       _stream()))

    def assemble_tangent(self, u, f_ext=None, vals=None, f_int=None, rhs=None, check=True):
        dev = self.device
        vals = torch.empty(self.nnz, dtype=torch.float64, device=dev) if vals is None else vals
        f_int = torch.empty(3 * self.model.mesh.n_nodes, dtype=torch.float64, device=dev) if f_int is None else f_int
        rhs = torch.empty(self.n_free, dtype=torch.float64, device=dev) if rhs is None else rhs
        du = _dev(u, torch.float64, dev)
        fe = None if f_ext is None else _dev(f_ext, torch.float64, dev)
        with torch.cuda.device(dev):
            _lib.check(self.lib.cxg_assemble_tangent(self.h, _ptr(du), _ptr(vals), _ptr(f_int), _ptr(rhs),
                                                     _ptr(fe), _stream()))
            if check:
                self.check()
        return vals, f_int, rhs

    def assemble_mass(self, density, lumped=False, vals=None, check=True):
        """Mass matrix M_ff on the plan's pattern (assemble_mass, src/fem/assembly.cpp:259-298);
        density per element."""
        vals = torch.empty(self.nnz, dtype=torch.float64, device=self.device) if vals is None else vals
        d = _dev(density, torch.float64, self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_assemble_mass(self.h, _ptr(d), int(bool(lumped)), _ptr(vals), _stream()))
            if check:
                self.check()
        return vals

    def assemble_geometric_stiffness(self, gp_stress, vals=None, check=True):
        """Initial-stress stiffness K_geo on the plan's pattern (assemble_geometric_stiffness,
        src/fem/assembly.cpp:300-331); gp_stress (n_gauss, 6) Voigt per Gauss point."""
        vals = torch.empty(self.nnz, dtype=torch.float64, device=self.device) if vals is None else vals
        sg = None if gp_stress is None else _dev(gp_stress, torch.float64, self.device).reshape(-1)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_assemble_geometric(self.h, _ptr(sg), _ptr(vals), _stream()))
            if check:
                self.check()
        return vals

    def recover_gauss_stress(self, u):
        """Gauss-point stress (n_gauss, 6) for the full displacement u (recover_gauss_stress,
        src/fem/stress.cpp:147-187)."""
        out = torch.empty(self.n_gauss * 6, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_recover_gauss_stress(self.h, _ptr(_dev(u, torch.float64, self.device)), _ptr(out),
                                                         _stream()))
            self.check()
        return out.view(-1, 6)

    def recover_fields(self, u, f_ext=None):
        """(nodal strain (N,6), nodal stress (N,6), reaction (N,3)) for the full
        displacement u (recover_fields, src/fem/stress.cpp:189-271)."""
        N = self.model.mesh.n_nodes
        st = torch.empty(6 * N, dtype=torch.float64, device=self.device)
        ss = torch.empty(6 * N, dtype=torch.float64, device=self.device)
        rf = torch.empty(3 * N, dtype=torch.float64, device=self.device)
        fe = None if f_ext is None else _dev(f_ext, torch.float64, self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_recover_fields(self.h, _ptr(_dev(u, torch.float64, self.device)), _ptr(fe),
                                                   _ptr(st), _ptr(ss), _ptr(rf), _stream()))
            self.check()
        return st.view(N, 6), ss.view(N, 6), rf.view(N, 3)

    # -- material state -------------------------------------------------------------
    def state(self, committed=True):
        out = torch.empty(self.n_gauss * 13, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_state_get(self.h, _lib.COMMITTED if committed else _lib.TRIAL, _ptr(out)))
        return out.view(self.n_gauss, 13)

    def set_state(self, state, committed=True):
        s = _dev(state, torch.float64, self.device).reshape(-1)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_state_set(self.h, _lib.COMMITTED if committed else _lib.TRIAL, _ptr(s)))

    def commit(self):
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_state_commit(self.h, _stream()))

    # -- reduced-system products, solve and adjoint ------------------------------------------
    def spmv(self, vals, x):
        y = torch.empty(self.n_free, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_spmv(self.h, _ptr(vals), _ptr(_dev(x, torch.float64, self.device)), _ptr(y),
                                         _stream()))
        return y

    def solve_cg(self, vals, rhs, x=None, rtol=1e-10, max_iter=20000):
        """K_ff x = rhs by Jacobi-preconditioned CG on the device (cxg_solve_cg)."""
        x = torch.zeros(self.n_free, dtype=torch.float64, device=self.device) if x is None else x
        it = C.c_int32()
        rel = C.c_double()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_solve_cg(self.h, _ptr(vals), _ptr(_dev(rhs, torch.float64, self.device)), _ptr(x),
                                             float(rtol), int(max_iter), C.byref(it), C.byref(rel), _stream()))
        return x, int(it.value), float(rel.value)

    def expand(self, x):
        """Full nodal displacement [3N] from the free solution: free DOFs from x, SPC
        DOFs at their prescribed value (linear_static.cpp:42-47 for SPC-only models)."""
        if not hasattr(self, "_free_idx"):
            self._free_idx = torch.as_tensor(np.nonzero(self.dof_eq >= 0)[0], device=self.device)
            self._pre = torch.as_tensor(self.prescribed, device=self.device)
        u = self._pre.clone()
        u[self._free_idx] = x
        return u

    def adjoint_compliance(self, u):
        """(dc/dE per element, dc/dX per node (N,3)) for c = f^T u (cxg_adjoint_compliance)."""
        m = self.model.mesh
        dE = torch.empty(m.n_elems, dtype=torch.float64, device=self.device)
        dX = torch.empty(3 * m.n_nodes, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_adjoint_compliance(self.h, _ptr(_dev(u, torch.float64, self.device)), _ptr(dE),
                                                       _ptr(dX), _stream()))
            self.check()
        return dE, dX.view(-1, 3)

    def update_coords(self, coords):
        c = _dev(coords, torch.float64, self.device)
        _lib.check(self.lib.cxg_plan_update_coords(self.h, _ptr(c)))

    def update_young(self, young):
        y = _dev(young, torch.float64, self.device)
        _lib.check(self.lib.cxg_plan_update_young(self.h, _ptr(y)))


# ---- the reference's function names ---------------------------------------------------

class ThermalPlan(Plan):
    """A temperature plan for heat conduction (assemble_conduction, src/fem/thermal.cpp:
    92-141): one DOF per node, prescribed temperatures tbc (node, value) eliminated."""

    def __init__(self, mesh, tbc_node=(), tbc_val=(), device=None):
        from .meshgen import thermal_dof_map
        self.lib = _lib.load()
        if not torch.cuda.is_available():
            raise _lib.CxgError(_lib.CXG_ERR_NO_GPU, "no CUDA device")
        self.device = torch.device(device or f"cuda:{torch.cuda.current_device()}")
        self.model = Model(mesh, [Material(1.0, 0.3)])
        deq, pre, nf = thermal_dof_map(mesh.n_nodes, tbc_node, tbc_val)
        self.t_dof_eq, self.t_prescribed, self.n_free = deq, pre, nf
        keep = []
        mats = (_lib.CxgMaterial * 1)(_c_material(Material(1.0, 0.3), keep))
        coords = _dev(mesh.coords, torch.float64, self.device)
        conn = _dev(mesh.conn.reshape(-1), torch.int32, self.device)
        desc = _lib.CxgMeshDesc(mesh.n_nodes, mesh.n_elems, mesh.etype, _ptr(coords), _ptr(conn), None, None, None, 1,
                                C.cast(mats, _vp))
        handle = _vp()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_thermal_plan_create(C.byref(desc), _vp(deq.ctypes.data), _vp(pre.ctypes.data), nf,
                                                        C.byref(handle)))
        self.h = handle
        info = _lib.CxgPlanInfo()
        _lib.check(self.lib.cxg_plan_get_info(self.h, C.byref(info)))
        self.info = info
        self.nnz = int(info.nnz)
        self.n_gauss = int(info.n_gauss_points)
        self._pattern = None

    def set_films(self, elem=(), face=(), h=(), sink=()):
        """*FILM faces (cxg_thermal_plan_set_films): element (0-based), face (1-based),
        coefficient and sink temperature per film; empty clears."""
        e = np.ascontiguousarray(elem, dtype=np.int64)
        f = np.ascontiguousarray(face, dtype=np.int32)
        hh = np.ascontiguousarray(h, dtype=np.float64)
        sk = np.ascontiguousarray(sink, dtype=np.float64)
        if not (e.size == f.size == hh.size == sk.size):
            raise ValueError("elem, face, h and sink must have one entry per film")
        ptr = lambda a: a.ctypes.data_as(C.c_void_p) if a.size else None
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_thermal_plan_set_films(self.h, e.size, ptr(e), ptr(f), ptr(hh), ptr(sk)))

    def assemble_conduction(self, conductivity, flux=None, vals=None, rhs=None, check=True):
        """(Kt_ff values, rhs = q_f - Kt_fc T_c); conductivity per element, flux per node."""
        dev = self.device
        vals = torch.empty(self.nnz, dtype=torch.float64, device=dev) if vals is None else vals
        rhs = torch.empty(self.n_free, dtype=torch.float64, device=dev) if rhs is None else rhs
        k = _dev(conductivity, torch.float64, dev)
        q = None if flux is None else _dev(flux, torch.float64, dev)
        with torch.cuda.device(dev):
            _lib.check(self.lib.cxg_assemble_conduction(self.h, _ptr(k), _ptr(q), _ptr(vals), _ptr(rhs), _stream()))
            if check:
                self.check()
        return vals, rhs


def assemble_linear_static(model: Model, precision: str = "fp64", plan: Plan | None = None) -> LinearSystem:
    """K_ff u_f = T^T f_ext - K_fc u_c (assembly.hpp:40-42)."""
    plan = plan or Plan(model, precision)
    vals, rhs = plan.assemble_linear(model.external_load_vector())
    rp, ci = plan.pattern()
    return LinearSystem(plan.n_free, rp, ci, vals, rhs, plan.dof_eq, plan.prescribed, {"plan": plan})


@dataclass
class MaterialPoints:
    """Per-Gauss-point history held on the device by a plan (assembly.hpp:76-88)."""

    plan: Plan

    def commit(self):
        self.plan.commit()

    def state(self, committed=True):
        return self.plan.state(committed)


def make_material_points(model: Model, precision: str = "fp64") -> MaterialPoints:
    return MaterialPoints(Plan(model, precision))


def assemble_material_tangent(model: Model, u, mp: MaterialPoints, f_int=None) -> LinearSystem:
    """Consistent tangent + internal force at the full displacement u (assembly.hpp:95-108).
    `u` is (N,3) or (3N,); f_int (torch, 3N) is filled when given."""
    plan = mp.plan
    vals, fi, rhs = plan.assemble_tangent(np.asarray(u, dtype=np.float64).reshape(-1) if not isinstance(u, torch.Tensor) else u.reshape(-1),
                                          model.external_load_vector(), f_int=f_int)
    rp, ci = plan.pattern()
    return LinearSystem(plan.n_free, rp, ci, vals, rhs, plan.dof_eq, plan.prescribed, {"f_int": fi})


def element_stiffness(etype: int, coords, E, nu, precision: str = "fp64") -> torch.Tensor:
    """Dense K_e for a batch of elements: coords (n,3) or (B,n,3); E, nu scalars or (B,)."""
    lib = _lib.load()
    dev = torch.device("cuda")
    x = _dev(coords, torch.float64, dev)
    single = x.dim() == 2
    x = x.reshape(-1, NODES[etype], 3)
    B = x.shape[0]
    Ev = _dev(np.broadcast_to(np.asarray(E, dtype=np.float64), (B,)).copy(), torch.float64, dev)
    nv = _dev(np.broadcast_to(np.asarray(nu, dtype=np.float64), (B,)).copy(), torch.float64, dev)
    nd = 3 * NODES[etype]
    Ke = torch.empty(B, nd, nd, dtype=torch.float64, device=dev)
    _lib.check(lib.cxg_element_stiffness(etype, B, _ptr(x), _ptr(Ev), _ptr(nv),
                                         _lib.MIXED if precision == "mixed" else _lib.FP64, _ptr(Ke), _stream()))
    return Ke[0] if single else Ke


def element_tangent_force(etype: int, coords, ue, material: Material, state=None, precision: str = "fp64"):
    """(Ke, fe, trial_state) for a batch: coords/ue (B,n,3); state (B,ngp,13) committed history."""
    lib = _lib.load()
    dev = torch.device("cuda")
    n, ngp = NODES[etype], NGP[etype]
    x = _dev(coords, torch.float64, dev)
    single = x.dim() == 2
    x = x.reshape(-1, n, 3)
    B = x.shape[0]
    u = _dev(ue, torch.float64, dev).reshape(B, n, 3)
    sc = None if state is None else _dev(state, torch.float64, dev).reshape(B, ngp, 13)
    st = torch.empty(B, ngp, 13, dtype=torch.float64, device=dev)
    nd = 3 * n
    Ke = torch.empty(B, nd, nd, dtype=torch.float64, device=dev)
    fe = torch.empty(B, nd, dtype=torch.float64, device=dev)
    keep = []
    cm = _c_material(material, keep)
    _lib.check(lib.cxg_element_tangent_force(etype, B, _ptr(x), _ptr(u), C.byref(cm), _ptr(sc), _ptr(st),
                                             _lib.MIXED if precision == "mixed" else _lib.FP64, _ptr(Ke),
                                             _ptr(fe), _stream()))
    if single:
        return Ke[0], fe[0], st[0]
    return Ke, fe, st
