"""The oracle against the committed golden vectors generated from the reference itself
(tests/golden/make_golden.py): bit-exact on element matrices, J2 updates and the
assembled cantilever; the reference's design sensitivity is stored for the adjoint."""
import hashlib
import os

import numpy as np
import pytest

from calculixpp_b200 import meshgen as mg
from calculixpp_b200.assembly import Material, Model
from oracle.oracle import make_material
from tests.helpers import ALL_TYPES, ISO_TABLE, box_model, per_element_materials

GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_vectors.npz"))


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_element_vectors(port, etype):
    x = GOLD[f"coords_{etype}"]
    assert np.array_equal(port.element_stiffness(etype, x, 195000.0, 0.28), GOLD[f"Ke_{etype}"])
    mat = make_material(210000.0, 0.3, ISO_TABLE)
    ue = GOLD[f"ue_{etype}"]
    K1, f1, s1 = port.element_tangent_force(etype, x, 0.5 * ue, mat)
    K2, f2, s2 = port.element_tangent_force(etype, x, ue, mat, s1.ravel())
    for got, key in ((K1, "KJ2a"), (f1, "fJ2a"), (s1, "sJ2a"), (K2, "KJ2b"), (f2, "fJ2b"), (s2, "sJ2b")):
        assert np.array_equal(got, GOLD[f"{key}_{etype}"]), key
    assert np.all(GOLD[f"sJ2b_{etype}"][:, 6] > 0)  # plastic branch


def test_cantilever_system(port):
    cfg = mg.cantilever_c3d8_config1()
    m, tip = cfg["mesh"], cfg["tip"]
    model = Model(m, [Material(210000.0, 0.3)], None, cfg["spc"],
                  (tip, np.full(tip.size, 2), np.full(tip.size, -1000.0 / tip.size)))
    dof_eq, pre, nf = model.dof_map()
    rp, ci, v, rhs = port.assemble_linear(m, [make_material(210000.0, 0.3)], None, dof_eq, pre, nf,
                                          model.external_load_vector())
    h = hashlib.sha256()
    h.update(rp.tobytes())
    h.update(ci.tobytes())
    assert h.hexdigest() == str(GOLD["cant_pattern_sha256"])
    assert v.size == int(GOLD["cant_nnz"])
    assert np.array_equal(rhs, GOLD["cant_rhs"])
    assert v.sum() == float(GOLD["cant_vals_sum"]) and (v * v).sum() == float(GOLD["cant_vals_sumsq"])
    rows = np.repeat(np.arange(nf), np.diff(rp))
    assert np.array_equal(v[rows == ci], GOLD["cant_vals_diag"])


def test_c3d20_box_system(port):
    box = box_model(mg.C3D20, 2, 2, 1, jitter=0.1, seed=77)
    assert np.array_equal(box.mesh.coords, GOLD["box20_coords"])
    mats, em = per_element_materials(box)
    dof_eq, pre, nf = box.dof_map()
    rp, ci, v, rhs = port.assemble_linear(box.mesh, mats, em, dof_eq, pre, nf, box.external_load_vector())
    assert np.array_equal(rp, GOLD["box20_row_ptr"]) and np.array_equal(ci, GOLD["box20_col_idx"])
    assert np.array_equal(v, GOLD["box20_vals"]) and np.array_equal(rhs, GOLD["box20_rhs"])


def test_sensitivity_vectors_consistent_with_element_fd(port):
    """The reference's semi-analytic compliance gradient equals the sum of per-element
    central differences -u_e^T dK_e/dX u_e of the oracle (same FD step 1e-4)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    sens = box_model(mg.C3D8, 4, 2, 2, jitter=0.05, seed=5)
    assert np.array_equal(sens.mesh.coords, GOLD["sens_coords"])
    mats, em = per_element_materials(sens)
    dof_eq, pre, nf = sens.dof_map()
    rp, ci, v, rhs = port.assemble_linear(sens.mesh, mats, em, dof_eq, pre, nf, sens.external_load_vector())
    uf = spla.spsolve(sp.csr_matrix((v, ci, rp), shape=(nf, nf)).tocsc(), rhs)
    assert abs(uf @ rhs - float(GOLD["sens_compliance"])) <= 1e-9 * abs(uf @ rhs)
    u = np.zeros(3 * sens.mesh.n_nodes)
    u[dof_eq >= 0] = uf
    g = np.zeros((sens.mesh.n_nodes, 3))
    m = sens.mesh
    for e in range(m.n_elems):
        c = m.conn[e]
        g[c] += port.element_compliance_grad_fd(m.etype, m.coords[c], u.reshape(-1, 3)[c], 210000.0, 0.3, 1e-4)
    gold = GOLD["sens_dcdX"]
    assert np.abs(g - gold).max() <= 1e-6 * np.abs(gold).max()
