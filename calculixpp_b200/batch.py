"""Batches of independent models (linear elastic or J2) assembled together (cxg_batch_*).

Models are grouped by element type inside libcxg; each group is one element pass and
one row gather over the concatenation of its models. Per model the results equal those
of a Plan of that model alone. The whole batch can run as one CUDA graph whose groups
are independent branches, and an autotuner picks each group's launch shape.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .assembly import Model, _c_material, _dev, _ptr, _stream

_vp = C.c_void_p
TILES = {0: "2x4", 1: "2x2", 2: "4x4"}


class Batch:
    """A cxg_batch on one GPU. `models` is a list of assembly.Model."""

    def __init__(self, models: list[Model], precision: str = "mixed", device=None):
        self.lib = _lib.load()
        if not torch.cuda.is_available():
            raise _lib.CxgError(_lib.CXG_ERR_NO_GPU, "no CUDA device")
        self.device = torch.device(device or f"cuda:{torch.cuda.current_device()}")
        self.models = models
        n = len(models)
        keep = []
        descs = (_lib.CxgMeshDesc * n)()
        dmaps = (_lib.CxgDofmapDesc * n)()
        for k, model in enumerate(models):
            m = model.mesh
            dof_eq, prescribed, n_free = model.dof_map()
            mats = (_lib.CxgMaterial * len(model.materials))(*[_c_material(x, keep) for x in model.materials])
            arrs = [np.ascontiguousarray(m.coords, dtype=np.float64),
                    np.ascontiguousarray(m.conn.reshape(-1), dtype=np.int32),
                    None if m.young is None else np.ascontiguousarray(m.young, dtype=np.float64),
                    None if m.poisson is None else np.ascontiguousarray(m.poisson, dtype=np.float64),
                    None if model.elem_mat is None else np.ascontiguousarray(model.elem_mat, dtype=np.int32),
                    np.ascontiguousarray(dof_eq, dtype=np.int32), np.ascontiguousarray(prescribed, dtype=np.float64)]
            keep += [mats] + [a for a in arrs if a is not None]
            p = [None if a is None else _vp(a.ctypes.data) for a in arrs]
            descs[k] = _lib.CxgMeshDesc(m.n_nodes, m.n_elems, m.etype, p[0], p[1], p[2], p[3], p[4],
                                        len(model.materials), C.cast(mats, _vp))
            dmaps[k] = _lib.CxgDofmapDesc(p[5], p[6], n_free)
        handle = _vp()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_batch_create(n, descs, dmaps, _lib.MIXED if precision == "mixed" else _lib.FP64,
                                                 C.byref(handle)))
        self.h = handle
        info = _lib.CxgBatchInfo()
        _lib.check(self.lib.cxg_batch_get_info(self.h, C.byref(info)))
        self.n_models, self.n_groups = int(info.n_models), int(info.n_groups)
        self.n_nodes, self.n_elems = int(info.n_nodes), int(info.n_elems)
        self.n_free, self.nnz = int(info.n_free), int(info.nnz)
        self.device_bytes = int(info.device_bytes)
        self.info = []
        for k in range(n):
            mi = _lib.CxgBatchModelInfo()
            _lib.check(self.lib.cxg_batch_get_model_info(self.h, k, C.byref(mi)))
            self.info.append(mi)

    # -- lifetime ----------------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.lib.cxg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- layout ------------------------------------------------------------------------
    def load_vector(self, loads=None):
        """Batch load vector in the batch's node order from per-model full vectors
        (None: each model's own CLOAD vector)."""
        f = np.zeros(3 * self.n_nodes)
        for k, model in enumerate(self.models):
            fk = model.external_load_vector() if loads is None else np.asarray(loads[k], dtype=np.float64)
            o = 3 * self.info[k].node_offset
            f[o:o + fk.size] = fk
        return f

    def slices(self, k, vals, rhs=None):
        mi = self.info[k]
        v = vals[mi.vals_offset:mi.vals_offset + mi.nnz]
        r = None if rhs is None else rhs[mi.rhs_offset:mi.rhs_offset + mi.n_free]
        return v, r

    def pattern(self, k):
        mi = self.info[k]
        rp = np.empty(mi.n_free + 1, dtype=np.int64)
        ci = np.empty(max(mi.nnz, 1), dtype=np.int32)
        _lib.check(self.lib.cxg_batch_get_pattern(self.h, k, _vp(rp.ctypes.data), _vp(ci.ctypes.data)))
        return rp, ci[:mi.nnz]

    def set_precision(self, precision: str):
        _lib.check(self.lib.cxg_batch_set_precision(self.h, _lib.MIXED if precision == "mixed" else _lib.FP64))

    LAUNCH_MODES = {"per_group": 0, "one_launch": 1}

    def set_launch(self, mode: str):
        """"per_group" (default): one element pass and one row gather per element-type
        group; "one_launch": one element pass and one row gather for the whole batch
        (cxg_batch_set_launch)."""
        _lib.check(self.lib.cxg_batch_set_launch(self.h, self.LAUNCH_MODES[mode]))

    def launch_mode(self) -> str:
        m = C.c_int32()
        _lib.check(self.lib.cxg_batch_get_launch(self.h, C.byref(m)))
        return {v: k for k, v in self.LAUNCH_MODES.items()}[m.value]

    def group_config(self, g):
        t, tile, p1, w = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        _lib.check(self.lib.cxg_batch_group_config(self.h, g, C.byref(t), C.byref(tile), C.byref(p1), C.byref(w)))
        return {"elem_type": t.value, "tile": TILES[tile.value], "p1_blocks_per_sm": p1.value, "p2_warps": w.value}

    def set_group_config(self, g, tile=0, p1_blocks_per_sm=0, p2_warps=0):
        _lib.check(self.lib.cxg_batch_set_group_config(self.h, g, tile, p1_blocks_per_sm, p2_warps))

    # -- work --------------------------------------------------------------------------
    def buffers(self):
        dev = self.device
        return (torch.empty(self.nnz, dtype=torch.float64, device=dev),
                torch.empty(self.n_free, dtype=torch.float64, device=dev))

    def assemble(self, f_ext=None, vals=None, rhs=None, check=True):
        if vals is None:
            vals, rhs = self.buffers()
        fe = None if f_ext is None else _dev(f_ext, torch.float64, self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_batch_assemble(self.h, _ptr(vals), _ptr(rhs), _ptr(fe), _stream()))
            if check:
                self.check()
        return vals, rhs

    def graph_launch(self, f_ext, vals, rhs, check=False):
        """Replay (capturing on first use for these buffers) the batch's CUDA graph;
        f_ext, vals and rhs must be device tensors."""
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_batch_graph_launch(self.h, _ptr(vals), _ptr(rhs), _ptr(f_ext), _stream()))
            if check:
                self.check()
        return vals, rhs

    def tune(self, f_ext, vals, rhs, cache_path=None):
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_batch_tune(self.h, _ptr(vals), _ptr(rhs), _ptr(f_ext),
                                               None if cache_path is None else str(cache_path).encode(), _stream()))
        return [self.group_config(g) for g in range(self.n_groups)]

    def check(self):
        _lib.check(self.lib.cxg_batch_check(self.h))

    # -- material-point (J2) assembly ------------------------------------------------------
    def displacement_vector(self, us):
        """Batch displacement vector (batch node order) from per-model full vectors."""
        u = np.zeros(3 * self.n_nodes)
        for k, uk in enumerate(us):
            o = 3 * self.info[k].node_offset
            uk = np.asarray(uk, dtype=np.float64).reshape(-1)
            u[o:o + uk.size] = uk
        return u

    def assemble_tangent(self, u, f_ext=None, vals=None, f_int=None, rhs=None, check=True):
        """Consistent tangent, internal force and rhs of every model at once
        (cxg_batch_assemble_tangent); u in batch node order (device or host array)."""
        dev = self.device
        if vals is None:
            vals, rhs = self.buffers()
        f_int = torch.empty(3 * self.n_nodes, dtype=torch.float64, device=dev) if f_int is None else f_int
        du = _dev(u, torch.float64, dev)
        fe = None if f_ext is None else _dev(f_ext, torch.float64, dev)
        with torch.cuda.device(dev):
            _lib.check(self.lib.cxg_batch_assemble_tangent(self.h, _ptr(du), _ptr(vals), _ptr(f_int), _ptr(rhs),
                                                           _ptr(fe), _stream()))
            if check:
                self.check()
        return vals, f_int, rhs

    def commit(self):
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_batch_commit(self.h, _stream()))

    def state(self, k, committed=True):
        """Model k's history (Gauss points, 13)."""
        mi = self.info[k]
        ng = mi.n_elems * _lib.load().cxg_gauss_points_per_element(self.models[k].mesh.etype)
        out = torch.empty(ng * 13, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.cxg_batch_get_state(self.h, k, _lib.COMMITTED if committed else _lib.TRIAL,
                                                    _ptr(out)))
        return out.view(ng, 13)

    def f_int_slice(self, k, f_int):
        o = 3 * self.info[k].node_offset
        return f_int[o:o + 3 * self.models[k].mesh.n_nodes]
