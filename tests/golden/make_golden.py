"""Generates tests/golden/reference_vectors.npz from the reference itself.

Runs the reference's own code (oracle/_ref/libcxpp_ref.so, compiled from its sources by
oracle/Makefile) on seeded inputs and stores its outputs:
  * element_stiffness for each family on one distorted element,
  * element_tangent_force with J2 isotropic hardening on the plastic branch (two
    increments, the second from the committed history of the first),
  * assemble_linear_static of the C3D8 cantilever (20x4x4 hexes of a 100x10x10 box):
    the CSR pattern digest, the rhs, and value checksums,
  * assemble_linear_static of a jittered 2x2x1 C3D20 box (full CSR),
  * the compliance design sensitivity (solve_sensitivity) of a 4x2x2 C3D8 cantilever
    for every node coordinate.

    python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from calculixpp_b200 import meshgen as mg  # noqa: E402
from calculixpp_b200.assembly import Material, Model  # noqa: E402
from oracle.oracle import Ref, coo_to_csr, make_material  # noqa: E402
from tests.helpers import ALL_TYPES, ISO_TABLE, box_model, distorted_elements, per_element_materials  # noqa: E402


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main():
    ref = Ref()
    out = {}
    for t in ALL_TYPES:
        x = distorted_elements(t, 1, seed=1000 + t, amp=0.1)[0]
        out[f"coords_{t}"] = x
        out[f"Ke_{t}"] = ref.element_stiffness(t, x, 195000.0, 0.28)
        mat = make_material(210000.0, 0.3, ISO_TABLE)
        G = np.random.default_rng(t).uniform(-0.012, 0.012, (3, 3))
        ue = x @ G.T
        out[f"ue_{t}"] = ue
        K1, f1, s1 = ref.element_tangent_force(t, x, 0.5 * ue, mat)
        K2, f2, s2 = ref.element_tangent_force(t, x, ue, mat, s1.ravel())
        out[f"KJ2a_{t}"], out[f"fJ2a_{t}"], out[f"sJ2a_{t}"] = K1, f1, s1
        out[f"KJ2b_{t}"], out[f"fJ2b_{t}"], out[f"sJ2b_{t}"] = K2, f2, s2

    cfg = mg.cantilever_c3d8_config1()
    m, tip = cfg["mesh"], cfg["tip"]
    model = Model(m, [Material(210000.0, 0.3)], None, cfg["spc"],
                  (tip, np.full(tip.size, 2), np.full(tip.size, -1000.0 / tip.size)))
    s = ref.model(m, [make_material(210000.0, 0.3)], None, model.spc, model.cloads).assemble_linear_static()
    rp, ci, v = coo_to_csr(s["n_free"], s["rows"], s["cols"], s["vals"])
    out["cant_pattern_sha256"] = np.array(digest(rp, ci))
    out["cant_nnz"] = np.array(v.size)
    out["cant_rhs"] = s["rhs"]
    out["cant_vals_sum"] = np.array(v.sum())
    out["cant_vals_sumsq"] = np.array((v * v).sum())
    rows = np.repeat(np.arange(s["n_free"]), np.diff(rp))
    out["cant_vals_diag"] = v[rows == ci]

    box = box_model(mg.C3D20, 2, 2, 1, jitter=0.1, seed=77)
    mats, em = per_element_materials(box)
    s = ref.model(box.mesh, mats, em, box.spc, box.cloads).assemble_linear_static()
    rp, ci, v = coo_to_csr(s["n_free"], s["rows"], s["cols"], s["vals"])
    out["box20_coords"] = box.mesh.coords
    out["box20_row_ptr"], out["box20_col_idx"], out["box20_vals"], out["box20_rhs"] = rp, ci, v, s["rhs"]

    sens = box_model(mg.C3D8, 4, 2, 2, jitter=0.05, seed=5)
    mats, em = per_element_materials(sens)
    rm = ref.model(sens.mesh, mats, em, sens.spc, sens.cloads)
    nodes = np.repeat(np.arange(sens.mesh.n_nodes), 3).astype(np.int32)
    comps = np.tile(np.arange(3), sens.mesh.n_nodes).astype(np.int32)
    dg, obj = rm.sensitivity_compliance(nodes, comps, h=1e-4)
    out["sens_coords"] = sens.mesh.coords
    out["sens_dcdX"] = dg.reshape(-1, 3)
    out["sens_compliance"] = np.array(obj)

    path = os.path.join(HERE, "reference_vectors.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
