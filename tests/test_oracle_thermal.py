"""Thermal strain in the oracle against the reference compiled from its sources.

*EXPANSION on the materials (a constant alpha and a temperature-dependent alpha(T) table)
with an applied temperature field on part of the nodes: thermal_strain_load_vector
(src/fem/loads.cpp:515-560), recover_gauss_stress and recover_fields with the thermal
correction (src/fem/stress.cpp:76-271) of the restatement equal the reference's bit for
bit, with the per-element alpha and t_ref from `thermal_strain_inputs` (the host side of
element_alpha).
"""
import numpy as np
import pytest

from calculixpp_b200 import meshgen as mg
from calculixpp_b200.thermal_strain import table_at, thermal_strain_inputs
from tests.helpers import ALL_TYPES, box_model, per_element_materials


def _thermal_case(etype, seed):
    quad = etype in (mg.C3D20, mg.C3D20R, mg.C3D15, mg.C3D10)
    dims = (2, 2, 1) if quad else (3, 2, 2)
    n_el = mg.box_mesh(etype, *dims).n_elems
    rng = np.random.default_rng(seed)
    model = box_model(etype, *dims, jitter=0.1, seed=seed, young=rng.uniform(70e3, 210e3, n_el))
    m = model.mesh
    mats, em = per_element_materials(model)
    # material k: constant alpha for even k, an alpha(T) table for odd k, t_ref 20 or 0
    tables, trefs, expansion = [], [], []
    for k in range(len(mats)):
        if k % 3 == 2:
            tables.append(None)
            trefs.append(0.0)
            expansion.append(None)
            continue
        if k % 2 == 0:
            vals, temps = [1.2e-5], [0.0]
        else:
            vals, temps = [1.0e-5, 1.3e-5, 1.7e-5], [0.0, 150.0, 400.0]
        tr = 20.0 if k % 2 == 0 else 0.0
        tables.append((vals, temps))
        trefs.append(tr)
        expansion.append((vals, temps, tr))
    T = rng.uniform(-50.0, 450.0, m.n_nodes)
    applied = (rng.uniform(size=m.n_nodes) < 0.7).astype(np.uint8)
    thermal = thermal_strain_inputs(m.conn, em, expansion, T, applied)
    return model, m, mats, em, tables, trefs, T, applied, thermal


def test_table_at_clamps_and_interpolates():
    v, t = [1.0, 3.0, 4.0], [0.0, 10.0, 20.0]
    assert table_at(v, t, -5.0) == 1.0 and table_at(v, t, 25.0) == 4.0
    assert table_at(v, t, 5.0) == 2.0 and table_at(v, t, 15.0) == 3.5
    assert table_at([7.0], [0.0], 100.0) == 7.0


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_thermal_strain_identical(port, ref, etype):
    model, m, mats, em, tables, trefs, T, applied, thermal = _thermal_case(etype, 40 + etype)
    rm = ref.model(m, mats, em, model.spc, model.cloads)
    rm.set_expansion(tables, trefs)
    on = np.flatnonzero(applied)
    rm.set_temperature(on, T[on])
    f_ref = rm.thermal_strain_load_vector()
    assert np.abs(f_ref).max() > 0.0
    assert np.array_equal(port.thermal_strain_load(m, m.young, m.poisson, thermal), f_ref)
    u = np.random.default_rng(etype + 9).uniform(-1e-3, 1e-3, 3 * m.n_nodes)
    assert np.array_equal(port.recover_gauss_stress_th(m, m.young, m.poisson, thermal, u), rm.recover_gauss_stress(u))
    a = port.recover_fields_th(m, m.young, m.poisson, thermal, u, model.external_load_vector())
    b = rm.recover_fields(u)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


N_FACES = {mg.C3D4: 4, mg.C3D10: 4, mg.C3D8: 6, mg.C3D8R: 6, mg.C3D20: 6, mg.C3D20R: 6, mg.C3D6: 5, mg.C3D15: 5}


def film_case(etype, seed):
    """Films on random element faces (some elements with two), prescribed temperatures on
    one face."""
    from tests.helpers import box_model as _box
    quad = etype in (mg.C3D20, mg.C3D20R, mg.C3D15, mg.C3D10)
    dims = (2, 2, 1) if quad else (3, 2, 2)
    model = _box(etype, *dims, jitter=0.1, seed=seed)
    m = model.mesh
    rng = np.random.default_rng(seed)
    elems = rng.choice(m.n_elems, size=min(m.n_elems, 6), replace=False)
    elems = np.concatenate([elems, elems[:2]])
    faces = rng.integers(1, N_FACES[etype] + 1, size=elems.size)
    h = rng.uniform(5.0, 50.0, elems.size)
    sink = rng.uniform(-20.0, 80.0, elems.size)
    hot = mg.face_nodes(m, 0, 0.0)
    tv = np.full(hot.size, 100.0)
    return model, m, (elems, faces, h, sink), hot, tv


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_conduction_films_identical(port, ref, etype):
    """assemble_conduction with *FILM faces (src/fem/thermal.cpp:113-126, face integrals of
    loads.cpp:361-389) of the restatement against the reference, bit for bit."""
    from calculixpp_b200.meshgen import thermal_dof_map
    from oracle.oracle import coo_to_csr
    model, m, films, tn, tv = film_case(etype, 90 + etype)
    mats, em = per_element_materials(model)
    k_mat = 40.0 + 5.0 * np.arange(len(mats))
    rm = ref.model(m, mats, em, model.spc, model.cloads)
    for e, f, h, s in zip(*films):
        rm.add_film(e, f, h, s)
    s = rm.assemble_conduction(k_mat, tn, tv)
    deq, pre, nf = thermal_dof_map(m.n_nodes, tn, tv)
    rp, ci, v = coo_to_csr(s["n_free"], s["rows"], s["cols"], s["vals"])
    rp2, ci2, v2, rhs2 = port.assemble_conduction_films(m, k_mat[em], deq, pre, nf, films)
    assert np.array_equal(rp, rp2) and np.array_equal(ci, ci2) and np.array_equal(v, v2)
    assert np.array_equal(s["rhs"], rhs2)
    _, _, v0, rhs0 = port.assemble_conduction(m, k_mat[em], deq, pre, nf)
    assert not np.array_equal(rhs0, rhs2)
