"""ctypes front end of the two CPU oracles. TEST INFRASTRUCTURE ONLY.

`Port`  wraps oracle/_lib/libcxo.so, the C restatement of the reference path (cxo.c).
`Ref`   wraps oracle/_ref/libcxpp_ref.so, the reference's own C++ sources compiled by
        oracle/Makefile with the shim in ref_shim.cpp (only present where the
        reference tree was available at build time).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module;
the product package never imports it. Both classes expose the same element-level
methods so a test can run one against the other.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_lib", "libcxo.so")
REF_SO = os.path.join(HERE, "_ref", "libcxpp_ref.so")
ADAPTER_SO = os.path.join(HERE, "_ref", "libcxg_cxpp_test.so")

NODES = {0: 4, 1: 10, 2: 8, 3: 8, 4: 20, 5: 20, 6: 6, 7: 15}
NGP = {0: 1, 1: 4, 2: 8, 3: 1, 4: 27, 5: 8, 6: 2, 7: 6}

_vp = C.c_void_p


class Material(C.Structure):
    """Layout shared by cxo_material, ref_material and cxg_material."""

    _fields_ = [("E", C.c_double), ("nu", C.c_double), ("n_plastic", C.c_int32),
                ("eqplastic", _vp), ("yield_", _vp), ("hardening", C.c_int32),
                ("h_kin", C.c_double)]


def make_material(E, nu, plastic=None, hardening=0, h_kin=0.0):
    """plastic: None (elastic) or (eqplastic[], yield[]). The returned object keeps its
    table arrays alive."""
    m = Material()
    m.E, m.nu, m.hardening, m.h_kin = float(E), float(nu), int(hardening), float(h_kin)
    if plastic is None:
        m.n_plastic, m.eqplastic, m.yield_ = 0, None, None
        m._keep = ()
    else:
        ep = np.ascontiguousarray(plastic[0], dtype=np.float64)
        sy = np.ascontiguousarray(plastic[1], dtype=np.float64)
        m.n_plastic = int(ep.size)
        m.eqplastic, m.yield_ = ep.ctypes.data, sy.ctypes.data
        m._keep = (ep, sy)
    return m


def _p(a):
    return None if a is None else a.ctypes.data_as(_vp)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


class OracleError(RuntimeError):
    pass


_i = C.c_int
_d = C.c_double
_i32t = C.c_int32
_i64t = C.c_int64

# Signatures of every entry point, (restype, argtypes). Handles come back as c_void_p so
# they keep all 64 bits; messages as c_char_p. Entries shared by both libraries first.
_COMMON = {
    "last_error": (C.c_char_p, []),
    "gauss_rule": (_i, [_i, _vp]),
    "shape": (_i, [_i, _d, _d, _d, _vp, _vp]),
    "physical_gradients": (_i, [_i, _d, _d, _d, _vp, _vp, _vp]),
    "element_volume": (_i, [_i, _vp, _vp]),
    "element_stiffness": (_i, [_i, _vp, _d, _d, _vp]),
    "material_evaluate": (_i, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "element_tangent_force": (_i, [_i, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "element_geometric_stiffness": (_i, [_i, _vp, _vp, _vp]),
    "element_conduction": (_i, [_i, _vp, _d, _vp]),
}

PORT_SIGS = dict(_COMMON, **{
    "nodes_per_element": (_i, [_i]),
    "dof_map": (_i32t, [_i64t, _i64t, _vp, _vp, _vp, _vp, _vp]),
    "assemble_linear": (_vp, [_i64t, _vp, _i64t, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32t, _vp]),
    "assemble_tangent": (_vp, [_i64t, _vp, _i64t, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32t, _vp, _vp, _vp,
                               _vp, _vp]),
    "element_mass": (_i, [_i, _vp, _d, _vp]),
    "element_mass_lumped": (_i, [_i, _vp, _d, _vp]),
    "assemble_scalar": (_vp, [_i, _i64t, _vp, _i64t, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32t]),
    "recover_gauss_stress": (_i, [_i64t, _vp, _i64t, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "recover_fields": (_i, [_i64t, _vp, _i64t, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "thermal_strain_load": (_i, [_i64t, _vp, _i64t, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "recover_gauss_stress_th": (_i, [_i64t, _vp, _i64t, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                     _vp]),
    "recover_fields_th": (_i, [_i64t, _vp, _i64t, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                               _vp, _vp, _vp]),
    "assemble_conduction": (_vp, [_i64t, _vp, _i64t, _vp, _vp, _vp, _vp, _vp, _vp, _i32t, _vp]),
    "assemble_conduction_films": (_vp, [_i64t, _vp, _i64t, _vp, _vp, _vp, _vp, _vp, _vp, _i32t, _vp, _i64t, _vp,
                                        _vp, _vp, _vp]),
    "system_info": (_i, [_vp, _vp, _vp]),
    "system_copy": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "system_free": (None, [_vp]),
    "element_compliance_grad_fd": (_i, [_i, _vp, _vp, _d, _d, _d, _vp]),
})

REF_SIGS = dict(_COMMON, **{
    "model_create": (_vp, [_i64t, _vp, _i64t, _vp, _vp, _vp, _vp, _i32t, _vp, _i64t, _vp, _vp, _vp, _i64t,
                           _vp, _vp, _vp]),
    "model_free": (None, [_vp]),
    "model_add_equation": (_i, [_vp, _i32t, _vp, _vp, _vp]),
    "element_mass": (_i, [_i, _vp, _d, _i, _vp]),
    "model_set_density": (_i, [_vp, _i32t, _vp]),
    "assemble_mass": (_vp, [_vp, _i]),
    "assemble_geometric": (_vp, [_vp, _vp]),
    "recover_gauss_stress": (_i, [_vp, _vp, _vp]),
    "recover_fields": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "model_set_expansion": (_i, [_vp, _i32t, _vp, _vp, _vp, _vp]),
    "model_set_temperature": (_i, [_vp, _i64t, _vp, _vp]),
    "model_add_film": (_i, [_vp, _i64t, _i32t, _d, _d]),
    "thermal_strain_load_vector": (_i, [_vp, _vp]),
    "assemble_conduction": (_vp, [_vp, _i32t, _vp, _i64t, _vp, _vp]),
    "assemble_linear_static": (_vp, [_vp]),
    "sys_info": (_i, [_vp, _vp, _vp]),
    "sys_copy": (_i, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "sys_free": (None, [_vp]),
    "mp_create": (_vp, [_vp]),
    "mp_free": (None, [_vp]),
    "mp_num_points": (_i64t, [_vp]),
    "mp_get_state": (_i, [_vp, _i, _vp]),
    "mp_set_state": (_i, [_vp, _i, _vp]),
    "mp_commit": (None, [_vp]),
    "assemble_material_tangent": (_vp, [_vp, _vp, _vp, _vp]),
    "sensitivity_compliance": (_i, [_vp, _i64t, _vp, _vp, _d, _vp, _vp]),
    "assemble_csr_threads": (_i, [_i, _vp, _i64t, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i]),
})


# The reference's drivers with the product's C++ adapter (ref_cuda_shim.cpp).
ADAPTER_SIGS = {
    "last_error": (C.c_char_p, []),
    "solve_linear_static": (_i, [_vp, _i, _i, _i, _vp, _vp]),
    "backend_solve": (_i, [_i32t, _i64t, _vp, _vp, _vp, _vp, _i, _vp]),
    "assembler_create": (_vp, [_vp, _i]),
    "assembler_free": (None, [_vp]),
    "assembler_sizes": (_i, [_vp, _vp, _vp]),
    "assemble_linear": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "assemble_tangent": (_i, [_vp, _i64t, _vp, _vp, _vp, _vp, _vp, _vp, _i]),
}


class _Base:
    prefix = ""
    sigs: dict = {}

    def __init__(self, path):
        if not os.path.exists(path):
            raise OracleError(f"oracle library missing: {path} (run make -C oracle)")
        self.lib = C.CDLL(path)
        # Every entry point is looked up once and configured once. CDLL.__getitem__
        # builds a new function object on each call, so settings made on one are lost;
        # the objects kept here carry their restype/argtypes for the library's lifetime.
        self._fns = {}
        for name, (res, args) in self.sigs.items():
            f = getattr(self.lib, f"{self.prefix}_{name}")
            f.restype = res
            f.argtypes = args
            self._fns[name] = f

    def _fn(self, name):
        try:
            return self._fns[name]
        except KeyError:
            raise OracleError(f"{self.prefix}_{name} has no declared signature") from None

    def last_error(self):
        msg = self._fn("last_error")()
        return msg.decode() if msg else ""

    def _check(self, rc):
        if rc != 0:
            raise OracleError(self.last_error())

    # ---- element level (same signatures in both libraries) -----------------------
    def gauss_rule(self, etype):
        out = np.zeros(4 * 27)
        n = self._fn("gauss_rule")(int(etype), _p(out))
        return out[: 4 * n].reshape(n, 4)

    def shape(self, etype, xi, et, ze):
        N = np.zeros(20)
        dN = np.zeros(60)
        f = self._fn("shape")
        n = f(int(etype), xi, et, ze, _p(N), _p(dN))
        return N[:n].copy(), dN[: 3 * n].reshape(n, 3).copy()

    def physical_gradients(self, etype, xi, et, ze, coords):
        n = NODES[etype]
        g = np.zeros(3 * n)
        det = C.c_double()
        f = self._fn("physical_gradients")
        self._check(f(int(etype), xi, et, ze, _p(_f64(coords)), _p(g), C.byref(det)))
        return g.reshape(n, 3), det.value

    def element_volume(self, etype, coords):
        v = C.c_double()
        self._check(self._fn("element_volume")(int(etype), _p(_f64(coords)), C.byref(v)))
        return v.value

    def element_stiffness(self, etype, coords, E, nu):
        n = NODES[etype]
        Ke = np.zeros((3 * n) * (3 * n))
        f = self._fn("element_stiffness")
        self._check(f(int(etype), _p(_f64(coords)), float(E), float(nu), _p(Ke)))
        return Ke.reshape(3 * n, 3 * n)

    def element_mass(self, etype, coords, rho, lumped=False):
        """element_mass / element_mass_lumped (element.hpp:93-102)."""
        n = NODES[etype]
        M = np.zeros((3 * n) ** 2)
        if self.prefix == "ref":
            f = self._fn("element_mass")
            self._check(f(int(etype), _p(_f64(coords)), float(rho), int(lumped), _p(M)))
        else:
            f = self._fn("element_mass_lumped" if lumped else "element_mass")
            self._check(f(int(etype), _p(_f64(coords)), float(rho), _p(M)))
        return M.reshape(3 * n, 3 * n)

    def element_geometric_stiffness(self, etype, coords, gp_stress):
        """element_geometric_stiffness (element.hpp:117-119); gp_stress (points, 6)."""
        n = NODES[etype]
        K = np.zeros((3 * n) ** 2)
        f = self._fn("element_geometric_stiffness")
        self._check(f(int(etype), _p(_f64(coords)), _p(_f64(gp_stress)), _p(K)))
        return K.reshape(3 * n, 3 * n)

    def element_conduction(self, etype, coords, k):
        """element_conduction (element.hpp:73-74): (n, n)."""
        n = NODES[etype]
        K = np.zeros(n * n)
        f = self._fn("element_conduction")
        self._check(f(int(etype), _p(_f64(coords)), float(k), _p(K)))
        return K.reshape(n, n)

    def material_evaluate(self, mat, strain, committed=None):
        committed = np.zeros(13) if committed is None else _f64(committed)
        trial = np.zeros(13)
        s = np.zeros(6)
        D = np.zeros(36)
        self._check(self._fn("material_evaluate")(C.byref(mat), _p(_f64(strain)),
                                                  _p(committed), _p(trial), _p(s), _p(D)))
        return s, D.reshape(6, 6), trial

    def element_tangent_force(self, etype, coords, ue, mat, committed=None):
        n = NODES[etype]
        ng = NGP[etype]
        committed = np.zeros(13 * ng) if committed is None else _f64(committed)
        trial = np.zeros(13 * ng)
        Ke = np.zeros((3 * n) ** 2)
        fe = np.zeros(3 * n)
        self._check(self._fn("element_tangent_force")(
            int(etype), _p(_f64(coords)), _p(_f64(ue)), C.byref(mat), _p(committed),
            _p(trial), _p(Ke), _p(fe)))
        return Ke.reshape(3 * n, 3 * n), fe, trial.reshape(ng, 13)


class Port(_Base):
    """The C restatement (oracle/cxo.c)."""

    prefix = "cxo"
    sigs = PORT_SIGS

    def __init__(self, path=PORT_SO):
        super().__init__(path)

    def _system(self, s):
        if not s:
            raise OracleError(self.last_error())
        n_free = C.c_int32()
        nnz = C.c_int64()
        self._fn("system_info")(_vp(s), C.byref(n_free), C.byref(nnz))
        rp = np.zeros(n_free.value + 1, dtype=np.int64)
        ci = np.zeros(nnz.value, dtype=np.int32)
        v = np.zeros(nnz.value)
        rhs = np.zeros(n_free.value)
        self._fn("system_copy")(_vp(s), _p(rp), _p(ci), _p(v), _p(rhs))
        self._fn("system_free")(_vp(s))
        return rp, ci, v, rhs

    @staticmethod
    def _mesh_arrays(mesh, mats, elem_mat):
        E = mesh.n_elems
        n = mesh.conn.shape[1]
        types = np.full(E, mesh.etype, dtype=np.int32)
        conn_ptr = np.arange(E + 1, dtype=np.int64) * n
        conn = _i32(mesh.conn.ravel())
        arr = (Material * len(mats))(*mats)
        em = _i32(elem_mat if elem_mat is not None else np.zeros(E, dtype=np.int32))
        return types, conn_ptr, conn, arr, em

    def assemble_linear(self, mesh, mats, elem_mat, dof_eq, prescribed, n_free, f_ext=None):
        """Reduced K_ff (canonical CSR) and rhs = T^T f_ext - K_fc u_c."""
        types, conn_ptr, conn, arr, em = self._mesh_arrays(mesh, mats, elem_mat)
        f = self._fn("assemble_linear")
        s = f(C.c_int64(mesh.n_nodes), _p(_f64(mesh.coords)), C.c_int64(mesh.n_elems),
              _p(types), _p(conn_ptr), _p(conn), _p(em), arr, _p(_i32(dof_eq)),
              _p(_f64(prescribed)), C.c_int32(n_free),
              _p(None if f_ext is None else _f64(f_ext)))
        return self._system(s)

    def assemble_tangent(self, mesh, mats, elem_mat, dof_eq, prescribed, n_free, u,
                         committed, f_ext=None):
        types, conn_ptr, conn, arr, em = self._mesh_arrays(mesh, mats, elem_mat)
        committed = _f64(committed)
        trial = np.zeros_like(committed)
        f_int = np.zeros(3 * mesh.n_nodes)
        f = self._fn("assemble_tangent")
        s = f(C.c_int64(mesh.n_nodes), _p(_f64(mesh.coords)), C.c_int64(mesh.n_elems),
              _p(types), _p(conn_ptr), _p(conn), _p(em), arr, _p(_i32(dof_eq)),
              _p(_f64(prescribed)), C.c_int32(n_free),
              _p(None if f_ext is None else _f64(f_ext)), _p(_f64(u)), _p(committed),
              _p(trial), _p(f_int))
        rp, ci, v, rhs = self._system(s)
        return rp, ci, v, rhs, f_int, trial

    def assemble_scalar(self, kind, mesh, dof_eq, prescribed, n_free, density=None, gp_stress=None):
        """assemble_mass (kind "mass" / "lumped") or assemble_geometric_stiffness
        (kind "geometric") as canonical CSR (rp, ci, vals); density per element,
        gp_stress (G, 6) in element order."""
        E = mesh.n_elems
        n = mesh.conn.shape[1]
        types = np.full(E, mesh.etype, dtype=np.int32)
        conn_ptr = np.arange(E + 1, dtype=np.int64) * n
        f = self._fn("assemble_scalar")
        code = {"mass": 1, "lumped": 2, "geometric": 3}[kind]
        s = f(code, mesh.n_nodes, _p(_f64(mesh.coords)), E, _p(types), _p(conn_ptr), _p(_i32(mesh.conn.ravel())),
              _p(None if density is None else _f64(density)), _p(None if gp_stress is None else _f64(gp_stress)),
              _p(_i32(dof_eq)), _p(_f64(prescribed)), int(n_free))
        rp, ci, v, _ = self._system(s)
        return rp, ci, v

    def _recover_args(self, mesh, young, poisson):
        E = mesh.n_elems
        n = mesh.conn.shape[1]
        return (mesh.n_nodes, _p(_f64(mesh.coords)), E, _p(np.full(E, mesh.etype, dtype=np.int32)),
                _p(np.arange(E + 1, dtype=np.int64) * n), _p(_i32(mesh.conn.ravel())), _p(_f64(young)),
                _p(_f64(poisson)))

    def recover_gauss_stress(self, mesh, young, poisson, u):
        """recover_gauss_stress (src/fem/stress.cpp:147-187): (G, 6)."""
        out = np.zeros(6 * mesh.n_elems * NGP[mesh.etype])
        f = self._fn("recover_gauss_stress")
        self._check(f(*self._recover_args(mesh, young, poisson), _p(_f64(u)), _p(out)))
        return out.reshape(-1, 6)

    def recover_fields(self, mesh, young, poisson, u, f_ext=None):
        """recover_fields (stress.cpp:189-271): nodal strain (N,6), stress (N,6), reaction (N,3)."""
        N = mesh.n_nodes
        st, ss, rf = np.zeros(6 * N), np.zeros(6 * N), np.zeros(3 * N)
        f = self._fn("recover_fields")
        self._check(f(*self._recover_args(mesh, young, poisson), _p(_f64(u)),
                      _p(None if f_ext is None else _f64(f_ext)), _p(st), _p(ss), _p(rf)))
        return st.reshape(N, 6), ss.reshape(N, 6), rf.reshape(N, 3)

    @staticmethod
    def _thermal_args(thermal):
        """(node_temp, node_applied, elem_alpha, elem_tref) pointers; thermal None: none."""
        if thermal is None:
            return (None, None, None, None), ()
        t, applied, alpha, tref = thermal
        keep = (_f64(t), None if applied is None else np.ascontiguousarray(applied, dtype=np.uint8), _f64(alpha),
                _f64(tref))
        return tuple(_p(k) for k in keep), keep

    def thermal_strain_load(self, mesh, young, poisson, thermal):
        """thermal_strain_load_vector (src/fem/loads.cpp:515-560): f[3N]. thermal = (node_temp,
        node_applied or None, elem_alpha, elem_tref)."""
        out = np.zeros(3 * mesh.n_nodes)
        ptrs, _keep = self._thermal_args(thermal)
        self._check(self._fn("thermal_strain_load")(*self._recover_args(mesh, young, poisson), *ptrs, _p(out)))
        return out

    def recover_gauss_stress_th(self, mesh, young, poisson, thermal, u):
        """recover_gauss_stress with the thermal-strain correction (stress.cpp:147-187): (G, 6)."""
        out = np.zeros(6 * mesh.n_elems * NGP[mesh.etype])
        ptrs, _keep = self._thermal_args(thermal)
        self._check(self._fn("recover_gauss_stress_th")(*self._recover_args(mesh, young, poisson), *ptrs,
                                                         _p(_f64(u)), _p(out)))
        return out.reshape(-1, 6)

    def recover_fields_th(self, mesh, young, poisson, thermal, u, f_ext=None):
        """recover_fields with thermal strain (stress.cpp:189-271): strain, stress, reaction."""
        N = mesh.n_nodes
        st, ss, rf = np.zeros(6 * N), np.zeros(6 * N), np.zeros(3 * N)
        ptrs, _keep = self._thermal_args(thermal)
        self._check(self._fn("recover_fields_th")(*self._recover_args(mesh, young, poisson), *ptrs, _p(_f64(u)),
                                                   _p(None if f_ext is None else _f64(f_ext)), _p(st), _p(ss),
                                                   _p(rf)))
        return st.reshape(N, 6), ss.reshape(N, 6), rf.reshape(N, 3)

    def assemble_conduction(self, mesh, conductivity, t_dof_eq, t_prescribed, n_free, flux=None):
        """assemble_conduction without films (src/fem/thermal.cpp:92-141): (rp, ci, vals, rhs)."""
        E = mesh.n_elems
        n = mesh.conn.shape[1]
        f = self._fn("assemble_conduction")
        s = f(mesh.n_nodes, _p(_f64(mesh.coords)), E, _p(np.full(E, mesh.etype, dtype=np.int32)),
              _p(np.arange(E + 1, dtype=np.int64) * n), _p(_i32(mesh.conn.ravel())), _p(_f64(conductivity)),
              _p(_i32(t_dof_eq)), _p(_f64(t_prescribed)), int(n_free), _p(None if flux is None else _f64(flux)))
        return self._system(s)

    def assemble_conduction_films(self, mesh, conductivity, t_dof_eq, t_prescribed, n_free, films, flux=None):
        """assemble_conduction with *FILM faces (thermal.cpp:92-141); films = (elem, face,
        h, sink) arrays, elements 0-based, faces 1-based: (rp, ci, vals, rhs)."""
        E = mesh.n_elems
        n = mesh.conn.shape[1]
        fe = np.ascontiguousarray(films[0], dtype=np.int64)
        ff, fh, fs = _i32(films[1]), _f64(films[2]), _f64(films[3])
        f = self._fn("assemble_conduction_films")
        s = f(mesh.n_nodes, _p(_f64(mesh.coords)), E, _p(np.full(E, mesh.etype, dtype=np.int32)),
              _p(np.arange(E + 1, dtype=np.int64) * n), _p(_i32(mesh.conn.ravel())), _p(_f64(conductivity)),
              _p(_i32(t_dof_eq)), _p(_f64(t_prescribed)), int(n_free), _p(None if flux is None else _f64(flux)),
              fe.size, _p(fe), _p(ff), _p(fh), _p(fs))
        return self._system(s)

    def element_compliance_grad_fd(self, etype, coords, ue, E, nu, h):
        n = NODES[etype]
        out = np.zeros(3 * n)
        f = self._fn("element_compliance_grad_fd")
        self._check(f(int(etype), _p(_f64(coords)), _p(_f64(ue)), E, nu, h, _p(out)))
        return out.reshape(n, 3)


def coo_to_csr(n, rows, cols, vals):
    """Canonical CSR (rows asc, cols asc, duplicates summed in input order)."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    key = rows * n + cols
    order = np.argsort(key, kind="stable")
    key = key[order]
    v = np.asarray(vals)[order]
    uniq, start = np.unique(key, return_index=True)
    sums = np.add.reduceat(v, start) if v.size else v
    r = (uniq // n).astype(np.int64)
    c = (uniq % n).astype(np.int32)
    rp = np.zeros(n + 1, dtype=np.int64)
    np.add.at(rp, r + 1, 1)
    return np.cumsum(rp), c, sums


class Ref(_Base):
    """The reference itself (oracle/_ref/libcxpp_ref.so)."""

    prefix = "ref"
    sigs = REF_SIGS

    def __init__(self, path=REF_SO):
        super().__init__(path)

    @staticmethod
    def available(path=REF_SO):
        return os.path.exists(path)

    def model(self, mesh, mats, elem_mat=None, spc=None, cloads=None):
        """Build a reference Model. spc=(node, comp, value) arrays, cloads likewise."""
        E = mesh.n_elems
        n = mesh.conn.shape[1]
        types = np.full(E, mesh.etype, dtype=np.int32)
        conn_ptr = np.arange(E + 1, dtype=np.int64) * n
        em = _i32(elem_mat if elem_mat is not None else np.zeros(E, dtype=np.int32))
        arr = (Material * len(mats))(*mats)
        sn, sc, sv = spc if spc is not None else (np.zeros(0), np.zeros(0), np.zeros(0))
        cn, cc, cv = cloads if cloads is not None else (np.zeros(0), np.zeros(0), np.zeros(0))
        sn, sc, sv, cn, cc, cv = _i32(sn), _i32(sc), _f64(sv), _i32(cn), _i32(cc), _f64(cv)
        h = self._fn("model_create")(
            C.c_int64(mesh.n_nodes), _p(_f64(mesh.coords)), C.c_int64(E), _p(types),
            _p(conn_ptr), _p(_i32(mesh.conn.ravel())), _p(em), C.c_int32(len(mats)), arr,
            C.c_int64(sn.size), _p(sn), _p(sc), _p(sv), C.c_int64(cn.size), _p(cn),
            _p(cc), _p(cv))
        if not h:
            raise OracleError(self.last_error())
        return RefModel(self, h, mesh)

    def _sys(self, s):
        if not s:
            raise OracleError(self.last_error())
        n_free = C.c_int64()
        nnz = C.c_int64()
        self._fn("sys_info")(_vp(s), C.byref(n_free), C.byref(nnz))
        rows = np.zeros(nnz.value, dtype=np.int32)
        cols = np.zeros(nnz.value, dtype=np.int32)
        vals = np.zeros(nnz.value)
        rhs = np.zeros(n_free.value)
        return n_free.value, rows, cols, vals, rhs, s

    def assemble_csr_threads(self, mesh, dof_eq, prescribed, row_ptr, col_idx, nthreads):
        vals = np.zeros(col_idx.size)
        rhs = np.zeros(row_ptr.size - 1)
        f = self._fn("assemble_csr_threads")
        self._check(f(int(mesh.etype), _p(_f64(mesh.coords)), mesh.n_elems,
                      _p(_i32(mesh.conn.ravel())), _p(_f64(mesh.young)),
                      _p(_f64(mesh.poisson)), _p(_i32(dof_eq)), _p(_f64(prescribed)),
                      _p(_i64(row_ptr)), _p(_i32(col_idx)), _p(vals), _p(rhs),
                      int(nthreads)))
        return vals, rhs


class RefModel:
    def __init__(self, ref, handle, mesh):
        self.ref, self.h, self.mesh = ref, handle, mesh
        self.mp = None

    def __del__(self):
        try:
            if self.mp:
                self.ref._fn("mp_free")(_vp(self.mp))
            self.ref._fn("model_free")(_vp(self.h))
        except Exception:
            pass

    def _take(self, s):
        n_free, rows, cols, vals, rhs, s = self.ref._sys(s)
        dof_eq = np.zeros(3 * self.mesh.n_nodes, dtype=np.int32)
        self.ref._fn("sys_copy")(_vp(s), _p(rows), _p(cols), _p(vals), _p(rhs), _p(dof_eq))
        self.ref._fn("sys_free")(_vp(s))
        return {"n_free": n_free, "rows": rows, "cols": cols, "vals": vals, "rhs": rhs,
                "dof_eq": dof_eq}

    def add_equation(self, nodes, comps, coeffs):
        """*EQUATION sum coeff_i u(node_i, comp_i) = 0, the first term dependent."""
        n, c, k = _i32(nodes), _i32(comps), _f64(coeffs)
        self.ref._check(self.ref._fn("model_add_equation")(_vp(self.h), n.size, _p(n), _p(c), _p(k)))

    def assemble_linear_static(self):
        """Returns the reference LinearSystem (COO in hash-map order) as a dict."""
        return self._take(self.ref._fn("assemble_linear_static")(_vp(self.h)))

    def time_linear_static(self, seconds):
        """Calls the reference's assemble_linear_static as shipped (one thread) until
        `seconds` have passed; returns (calls, elapsed seconds). The systems are freed
        untouched, so only the reference call is timed."""
        fn, free = self.ref._fn("assemble_linear_static"), self.ref._fn("sys_free")
        calls, t0 = 0, time.perf_counter()
        while True:
            free(_vp(fn(_vp(self.h))))
            calls += 1
            dt = time.perf_counter() - t0
            if dt >= seconds:
                return calls, dt

    def assemble_conduction(self, k_per_material, tbc_node, tbc_val):
        k = _f64(k_per_material)
        tn, tv = _i32(tbc_node), _f64(tbc_val)
        f = self.ref._fn("assemble_conduction")
        return self._take(f(_vp(self.h), k.size, _p(k), tn.size, _p(tn), _p(tv)))

    def recover_gauss_stress(self, u):
        out = np.zeros(6 * self.mesh.n_elems * NGP[self.mesh.etype])
        self.ref._check(self.ref._fn("recover_gauss_stress")(_vp(self.h), _p(_f64(u)), _p(out)))
        return out.reshape(-1, 6)

    def recover_fields(self, u):
        N = self.mesh.n_nodes
        st, ss, rf = np.zeros(6 * N), np.zeros(6 * N), np.zeros(3 * N)
        self.ref._check(self.ref._fn("recover_fields")(_vp(self.h), _p(_f64(u)), _p(st), _p(ss), _p(rf)))
        return st.reshape(N, 6), ss.reshape(N, 6), rf.reshape(N, 3)

    def set_expansion(self, tables, trefs):
        """*EXPANSION per material: tables[k] = (alpha values, temperatures) or None."""
        npts = np.array([0 if t is None else len(t[0]) for t in tables], dtype=np.int32)
        vals = _f64(np.concatenate([np.asarray(t[0], float) for t in tables if t is not None] or [np.zeros(0)]))
        temps = _f64(np.concatenate([np.asarray(t[1], float) for t in tables if t is not None] or [np.zeros(0)]))
        tr = _f64(trefs)
        self.ref._check(self.ref._fn("model_set_expansion")(_vp(self.h), C.c_int32(npts.size), _p(npts), _p(vals),
                                                             _p(temps), _p(tr)))

    def add_film(self, elem, face, h, sink):
        """A *FILM face (Model::films): element 0-based, face 1-based."""
        self.ref._check(self.ref._fn("model_add_film")(_vp(self.h), int(elem), int(face), float(h), float(sink)))

    def set_temperature(self, nodes, temps):
        """Applied temperatures (Model::applied_temperature), nodes 0-based."""
        nd, tv = _i32(nodes), _f64(temps)
        self.ref._check(self.ref._fn("model_set_temperature")(_vp(self.h), nd.size, _p(nd), _p(tv)))

    def thermal_strain_load_vector(self):
        out = np.zeros(3 * self.mesh.n_nodes)
        self.ref._check(self.ref._fn("thermal_strain_load_vector")(_vp(self.h), _p(out)))
        return out

    def set_density(self, rho_per_material):
        rho = _f64(rho_per_material)
        self.ref._check(self.ref._fn("model_set_density")(_vp(self.h), C.c_int32(rho.size), _p(rho)))

    def assemble_mass(self, lumped=False):
        f = self.ref._fn("assemble_mass")
        return self._take(f(_vp(self.h), int(lumped)))

    def assemble_geometric(self, gp_stress):
        f = self.ref._fn("assemble_geometric")
        return self._take(f(_vp(self.h), _p(_f64(gp_stress))))

    def material_points(self):
        if self.mp is None:
            self.mp = self.ref._fn("mp_create")(_vp(self.h))
            if not self.mp:
                raise OracleError(self.ref.last_error())
        return self.mp

    def state(self, committed=True):
        mp = self.material_points()
        g = self.ref._fn("mp_num_points")(_vp(mp))
        out = np.zeros(13 * g)
        self.ref._fn("mp_get_state")(_vp(mp), int(committed), _p(out))
        return out

    def set_state(self, state, committed=True):
        mp = self.material_points()
        self.ref._fn("mp_set_state")(_vp(mp), int(committed), _p(_f64(state)))

    def commit(self):
        self.ref._fn("mp_commit")(_vp(self.material_points()))

    def assemble_material_tangent(self, u):
        mp = self.material_points()
        f_int = np.zeros(3 * self.mesh.n_nodes)
        s = self.ref._fn("assemble_material_tangent")(_vp(self.h), _vp(mp),
                                                      _p(_f64(u)), _p(f_int))
        out = self._take(s)
        out["f_int"] = f_int
        return out

    def sensitivity_compliance(self, var_node, var_comp, h=1e-4):
        var_node, var_comp = _i32(var_node), _i32(var_comp)
        dg = np.zeros(var_node.size)
        obj = C.c_double()
        f = self.ref._fn("sensitivity_compliance")
        self.ref._check(f(_vp(self.h), var_node.size, _p(var_node), _p(var_comp), h,
                          _p(dg), C.byref(obj)))
        return dg, obj.value


class RefCuda(_Base):
    """The reference's linear-static driver and assembly calls with the assembly through
    the product's C++ adapter (oracle/_ref/libcxg_cxpp_test.so); models come from Ref."""

    prefix = "cuda"
    sigs = ADAPTER_SIGS

    def __init__(self, path=ADAPTER_SO):
        super().__init__(path)

    @staticmethod
    def available(path=ADAPTER_SO):
        return os.path.exists(path)

    def solve_linear_static(self, ref_model, gpu, precision=0, solver=0):
        """(u (N,3), nodal stress (N,6)) of numerics::solve_linear_static; gpu 0 all on
        the CPU, 1 the adapter's assembly, 2 the adapter's assembly and device solve;
        solver 0 direct, 1 CG."""
        N = ref_model.mesh.n_nodes
        u, st = np.zeros(3 * N), np.zeros(6 * N)
        self._check(self._fn("solve_linear_static")(_vp(ref_model.h), int(gpu), int(precision), int(solver), _p(u),
                                                    _p(st)))
        return u.reshape(N, 3), st.reshape(N, 6)

    def backend_solve(self, n, rows, cols, vals, rhs, solver=0):
        """CudaBackend::solve_sparse on COO triplets."""
        rows, cols, vals, rhs = _i32(rows), _i32(cols), _f64(vals), _f64(rhs)
        x = np.zeros(int(n))
        self._check(self._fn("backend_solve")(int(n), vals.size, _p(rows), _p(cols), _p(vals), _p(rhs), int(solver),
                                              _p(x)))
        return x

    def assembler(self, ref_model, precision=0):
        h = self._fn("assembler_create")(_vp(ref_model.h), int(precision))
        if not h:
            raise OracleError(self.last_error())
        return h

    def free(self, h):
        self._fn("assembler_free")(_vp(h))

    def _arrays(self, h):
        nnz, nf = C.c_int64(), C.c_int64()
        self._check(self._fn("assembler_sizes")(_vp(h), C.byref(nnz), C.byref(nf)))
        n = nnz.value
        return np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n), np.zeros(nf.value)

    def assemble_linear(self, h):
        """The adapter's LinearSystem: (rows, cols, vals, rhs), COO in (row, column) order."""
        rows, cols, vals, rhs = self._arrays(h)
        self._check(self._fn("assemble_linear")(_vp(h), _p(rows), _p(cols), _p(vals), _p(rhs)))
        return rows, cols, vals, rhs

    def assemble_tangent(self, h, u, commit=False):
        """assemble_material_tangent through the adapter at u[3N]: (rows, cols, vals, rhs,
        f_int); commit afterwards when asked."""
        u = _f64(u)
        rows, cols, vals, rhs = self._arrays(h)
        f_int = np.zeros(u.size)
        self._check(self._fn("assemble_tangent")(_vp(h), u.size // 3, _p(u), _p(rows), _p(cols), _p(vals), _p(rhs),
                                                 _p(f_int), int(commit)))
        return rows, cols, vals, rhs, f_int
