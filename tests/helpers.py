"""Shared builders and comparisons for the tests."""
from __future__ import annotations

import numpy as np

from calculixpp_b200 import meshgen as mg
from calculixpp_b200.assembly import Material, Model

ALL_TYPES = (mg.C3D8, mg.C3D8R, mg.C3D20, mg.C3D20R, mg.C3D6, mg.C3D15, mg.C3D4, mg.C3D10)

# Isotropic hardening table used by the reference's own plasticity tests
# (tests/test_plasticity.cpp:27-33): sy0 = 800 at ep = 0, sy = 960 at ep = 0.02.
ISO_TABLE = ([0.0, 0.02], [800.0, 960.0])


def unit_element(etype):
    """The reference tests' straight-edged unit hex / wedge (tests/test_element.cpp:146-193)."""
    m = mg.box_mesh(etype, 1, 1, 1)
    return m.coords[m.conn[0]].copy()


def distorted_elements(etype, count, seed=0, amp=0.08):
    """Unit elements with every node moved by uniform(-amp, amp) (positive Jacobians)."""
    rng = np.random.default_rng(seed)
    x0 = unit_element(etype)
    return x0[None] + rng.uniform(-amp, amp, size=(count,) + x0.shape)


def box_model(etype, nx, ny, nz, jitter=0.1, seed=0, young=None, materials=None, clamp_axis=0,
              load=True, prescribe=None):
    """Box mesh with one face clamped and a load (or a prescribed motion) on the opposite face."""
    m = mg.box_mesh(etype, nx, ny, nz, float(nx), float(ny), float(nz), jitter=jitter, seed=seed)
    E = m.n_elems
    m.young = np.full(E, 210000.0) if young is None else young
    m.poisson = np.full(E, 0.3)
    sn, sc, sv = mg.clamp_face_spc(m, clamp_axis, 0.0)
    far = mg.face_nodes(m, clamp_axis, float((nx, ny, nz)[clamp_axis]))
    cl = None
    if prescribe is not None:
        sn = np.concatenate([sn, far.astype(np.int32)])
        sc = np.concatenate([sc, np.full(far.size, clamp_axis, dtype=np.int32)])
        sv = np.concatenate([sv, np.full(far.size, prescribe)])
    elif load:
        cl = (far, np.full(far.size, 2), np.full(far.size, -1000.0 / far.size))
    mats = materials or [Material(210000.0, 0.3)]
    return Model(m, mats, None, (sn, sc, sv), cl)


def oracle_materials(model):
    from oracle.oracle import make_material
    out = []
    for mat in model.materials:
        out.append(make_material(mat.E, mat.nu, mat.plastic, mat.hardening, mat.h_kin))
    return out


def per_element_materials(model):
    """Reference/port material list + element map honouring per-element E/nu."""
    from oracle.oracle import make_material
    m = model.mesh
    base = model.elem_mat if model.elem_mat is not None else np.zeros(m.n_elems, dtype=np.int32)
    mats, index, em = [], {}, np.zeros(m.n_elems, dtype=np.int32)
    for e in range(m.n_elems):
        src = model.materials[int(base[e])]
        E = float(m.young[e]) if m.young is not None else src.E
        nu = float(m.poisson[e]) if m.poisson is not None else src.nu
        key = (E, nu, int(base[e]))
        if key not in index:
            index[key] = len(mats)
            mats.append(make_material(E, nu, src.plastic, src.hardening, src.h_kin))
        em[e] = index[key]
    return mats, em


def rel_fro(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def to_np(t):
    import torch
    return t.detach().cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)
