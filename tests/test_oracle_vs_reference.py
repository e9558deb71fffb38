"""Pins the oracle: the C restatement (oracle/cxo.c) against the reference itself
(oracle/_ref/libcxpp_ref.so, built from the reference's own sources), bit for bit.

Both are compiled with -ffp-contract=off and the restatement keeps the reference's
operation order, so element matrices, J2 updates and assembled systems are identical,
not merely close."""
import numpy as np
import pytest

from calculixpp_b200 import meshgen as mg
from oracle.oracle import coo_to_csr, make_material
from tests.helpers import ALL_TYPES, ISO_TABLE, box_model, distorted_elements, per_element_materials

MATS = [
    (210000.0, 0.3, None, 0, 0.0),
    (210000.0, 0.3, ISO_TABLE, 0, 0.0),
    (210000.0, 0.3, ISO_TABLE, 1, 0.0),
    (210000.0, 0.3, ISO_TABLE, 2, 5000.0),
    (210000.0, 0.3, ([0.0], [800.0]), 0, 0.0),
    (200000.0, 0.29, ([0.0, 0.01, 0.03], [300.0, 420.0, 500.0]), 0, 0.0),
]


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_gauss_and_shapes_identical(port, ref, etype):
    gp = port.gauss_rule(etype)
    assert np.array_equal(gp, ref.gauss_rule(etype))
    for q in range(gp.shape[0]):
        N1, d1 = port.shape(etype, *gp[q, :3])
        N2, d2 = ref.shape(etype, *gp[q, :3])
        assert np.array_equal(N1, N2) and np.array_equal(d1, d2)


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_element_stiffness_identical(port, ref, etype):
    for x in distorted_elements(etype, 6, seed=etype, amp=0.1):
        assert np.array_equal(port.element_stiffness(etype, x, 185000.0, 0.27),
                              ref.element_stiffness(etype, x, 185000.0, 0.27))
        assert port.element_volume(etype, x) == ref.element_volume(etype, x)


@pytest.mark.parametrize("etype", ALL_TYPES)
@pytest.mark.parametrize("mi", range(len(MATS)))
def test_element_tangent_force_identical(port, ref, etype, mi):
    mat = make_material(*MATS[mi])
    rng = np.random.default_rng(10 * etype + mi)
    ngp = mg.NGP[etype]
    for x in distorted_elements(etype, 4, seed=etype + 20):
        G = rng.uniform(-0.01, 0.01, (3, 3))
        committed = np.zeros(13 * ngp)
        for step in (1, 2):
            ue = (x @ G.T) * step
            a = port.element_tangent_force(etype, x, ue, mat, committed)
            b = ref.element_tangent_force(etype, x, ue, mat, committed)
            for u, v in zip(a, b):
                assert np.array_equal(u, v)
            committed = a[2].ravel()


def test_material_evaluate_identical(port, ref):
    rng = np.random.default_rng(7)
    for args in MATS:
        mat = make_material(*args)
        for _ in range(20):
            strain = rng.uniform(-0.01, 0.01, 6)
            committed = np.zeros(13)
            committed[6] = abs(rng.normal(0, 0.002))
            a = port.material_evaluate(mat, strain, committed)
            b = ref.material_evaluate(mat, strain, committed)
            for u, v in zip(a, b):
                assert np.array_equal(u, v)


def _ref_csr(model, ref):
    mats, em = per_element_materials(model)
    rm = ref.model(model.mesh, mats, em, model.spc, model.cloads)
    s = rm.assemble_linear_static()
    rp, ci, v = coo_to_csr(s["n_free"], s["rows"], s["cols"], s["vals"])
    return rm, s, rp, ci, v


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_assemble_linear_static_identical(port, ref, etype):
    quad = etype in (mg.C3D20, mg.C3D20R, mg.C3D15)
    dims = (2, 2, 1) if quad else (3, 2, 2)
    E = np.random.default_rng(etype).uniform(70e3, 210e3, mg.box_mesh(etype, *dims).n_elems)
    model = box_model(etype, *dims, jitter=0.1, seed=etype, young=E, prescribe=0.01 if etype == mg.C3D8 else None)
    rm, s, rp, ci, v = _ref_csr(model, ref)
    dof_eq, pre, nf = model.dof_map()
    assert np.array_equal(dof_eq, s["dof_eq"]) and nf == s["n_free"]
    mats, em = per_element_materials(model)
    rp2, ci2, v2, rhs2 = port.assemble_linear(model.mesh, mats, em, dof_eq, pre, nf, model.external_load_vector())
    assert np.array_equal(rp, rp2) and np.array_equal(ci, ci2)
    assert np.array_equal(v, v2)
    assert np.array_equal(s["rhs"], rhs2)


def test_config1_cantilever_identical(port, ref):
    cfg = mg.cantilever_c3d8_config1()
    m, tip = cfg["mesh"], cfg["tip"]
    from calculixpp_b200.assembly import Material, Model
    model = Model(m, [Material(210000.0, 0.3)], None, cfg["spc"],
                  (tip, np.full(tip.size, 2), np.full(tip.size, -1000.0 / tip.size)))
    rm, s, rp, ci, v = _ref_csr(model, ref)
    assert s["n_free"] == 1500 and v.size == 88218  # topological nnz, no exact zeros
    dof_eq, pre, nf = model.dof_map()
    rp2, ci2, v2, rhs2 = port.assemble_linear(m, [make_material(210000.0, 0.3)], None, dof_eq, pre, nf,
                                              model.external_load_vector())
    assert np.array_equal(rp, rp2) and np.array_equal(ci, ci2) and np.array_equal(v, v2)
    assert np.array_equal(s["rhs"], rhs2)


@pytest.mark.parametrize("etype", [mg.C3D8, mg.C3D8R, mg.C3D20R, mg.C3D15])
def test_assemble_material_tangent_identical(port, ref, etype):
    from calculixpp_b200.assembly import Material
    mat = Material(210000.0, 0.3, ([0.0, 1.0], [250.0, 1250.0]))
    dims = (2, 1, 1) if etype in (mg.C3D20R, mg.C3D15) else (3, 2, 1)
    model = box_model(etype, *dims, materials=[mat], load=False, prescribe=0.004)
    mats, em = per_element_materials(model)
    rm = ref.model(model.mesh, mats, em, model.spc, model.cloads)
    dof_eq, pre, nf = model.dof_map()
    committed = np.zeros(rm.state().size)
    rng = np.random.default_rng(etype)
    for k in (1, 2, 3):
        u = np.zeros(3 * model.mesh.n_nodes)
        u[dof_eq < 0] = pre[dof_eq < 0] * k / 3.0
        u[dof_eq >= 0] = rng.uniform(-2e-3, 2e-3, nf) * k
        s = rm.assemble_material_tangent(u)
        rp, ci, v = coo_to_csr(s["n_free"], s["rows"], s["cols"], s["vals"])
        rp2, ci2, v2, rhs2, f2, st2 = port.assemble_tangent(model.mesh, mats, em, dof_eq, pre, nf, u, committed)
        assert np.array_equal(rp, rp2) and np.array_equal(ci, ci2) and np.array_equal(v, v2)
        assert np.array_equal(s["rhs"], rhs2) and np.array_equal(s["f_int"], f2)
        assert np.array_equal(rm.state(committed=False), st2)
        rm.commit()
        committed = st2
    assert np.any(committed.reshape(-1, 13)[:, 6] > 0)


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_element_mass_and_geometric_identical(port, ref, etype):
    rng = np.random.default_rng(300 + etype)
    for x in distorted_elements(etype, 4, seed=etype + 40, amp=0.1):
        for lumped in (False, True):
            assert np.array_equal(port.element_mass(etype, x, 7.85e-9, lumped),
                                  ref.element_mass(etype, x, 7.85e-9, lumped))
        s = rng.normal(0.0, 100.0, (mg.NGP[etype], 6))
        assert np.array_equal(port.element_geometric_stiffness(etype, x, s),
                              ref.element_geometric_stiffness(etype, x, s))


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_assemble_mass_and_geometric_identical(port, ref, etype):
    """assemble_mass (consistent and lumped) and assemble_geometric_stiffness
    (src/fem/assembly.cpp:259-331) against the reference's own drivers."""
    quad = etype in (mg.C3D20, mg.C3D20R, mg.C3D15)
    dims = (2, 2, 1) if quad else (3, 2, 2)
    n_el = mg.box_mesh(etype, *dims).n_elems
    E = np.random.default_rng(etype).uniform(70e3, 210e3, n_el)
    model = box_model(etype, *dims, jitter=0.1, seed=etype, young=E, prescribe=0.01)
    mats, em = per_element_materials(model)
    rho_mat = 7.85e-9 * (1.0 + 0.1 * np.arange(len(mats)))
    rm = ref.model(model.mesh, mats, em, model.spc, model.cloads)
    rm.set_density(rho_mat)
    dof_eq, pre, nf = model.dof_map()
    gs = np.random.default_rng(etype + 1).normal(0.0, 50.0, (n_el * mg.NGP[etype], 6))
    for kind in ("mass", "lumped", "geometric"):
        s = rm.assemble_geometric(gs) if kind == "geometric" else rm.assemble_mass(kind == "lumped")
        rp, ci, v = coo_to_csr(s["n_free"], s["rows"], s["cols"], s["vals"])
        rp2, ci2, v2 = port.assemble_scalar(kind, model.mesh, dof_eq, pre, nf, density=rho_mat[em], gp_stress=gs)
        assert np.array_equal(rp, rp2) and np.array_equal(ci, ci2), kind
        assert np.array_equal(v, v2), kind
        assert not np.any(s["rhs"]), kind


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_recover_stress_and_fields_identical(port, ref, etype):
    """recover_gauss_stress and recover_fields (src/fem/stress.cpp:147-271) of the
    restatement against the reference, for a displacement field with a load."""
    quad = etype in (mg.C3D20, mg.C3D20R, mg.C3D15)
    dims = (2, 2, 1) if quad else (3, 2, 2)
    n_el = mg.box_mesh(etype, *dims).n_elems
    E = np.random.default_rng(etype).uniform(70e3, 210e3, n_el)
    model = box_model(etype, *dims, jitter=0.1, seed=etype, young=E)
    m = model.mesh
    mats, em = per_element_materials(model)
    rm = ref.model(m, mats, em, model.spc, model.cloads)
    u = np.random.default_rng(etype + 7).uniform(-1e-3, 1e-3, 3 * m.n_nodes)
    assert np.array_equal(port.recover_gauss_stress(m, m.young, m.poisson, u), rm.recover_gauss_stress(u))
    a = port.recover_fields(m, m.young, m.poisson, u, model.external_load_vector())
    b = rm.recover_fields(u)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_conduction_identical(port, ref, etype):
    """element_conduction and assemble_conduction (src/fem/thermal.cpp:92-141) with
    prescribed temperatures on one face, against the reference."""
    for x in distorted_elements(etype, 3, seed=etype + 60, amp=0.1):
        assert np.array_equal(port.element_conduction(etype, x, 45.0), ref.element_conduction(etype, x, 45.0))
    quad = etype in (mg.C3D20, mg.C3D20R, mg.C3D15, mg.C3D10)
    dims = (2, 2, 1) if quad else (3, 2, 2)
    model = box_model(etype, *dims, jitter=0.1, seed=etype)
    m = model.mesh
    mats, em = per_element_materials(model)
    k_mat = 40.0 + 5.0 * np.arange(len(mats))
    hot = mg.face_nodes(m, 0, 0.0)
    cold = mg.face_nodes(m, 0, float(dims[0]))
    tn = np.concatenate([hot, cold])
    tv = np.concatenate([np.full(hot.size, 100.0), np.full(cold.size, 20.0)])
    rm = ref.model(m, mats, em, model.spc, model.cloads)
    s = rm.assemble_conduction(k_mat, tn, tv)
    deq, pre, nf = mg.thermal_dof_map(m.n_nodes, tn, tv)
    assert np.array_equal(s["dof_eq"][:m.n_nodes], deq) and s["n_free"] == nf
    rp, ci, v = coo_to_csr(s["n_free"], s["rows"], s["cols"], s["vals"])
    rp2, ci2, v2, rhs2 = port.assemble_conduction(m, k_mat[em], deq, pre, nf)
    assert np.array_equal(rp, rp2) and np.array_equal(ci, ci2) and np.array_equal(v, v2)
    assert np.array_equal(s["rhs"], rhs2)
