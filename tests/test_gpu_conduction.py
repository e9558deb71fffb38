"""Heat-conduction assembly through the CUDA path against the oracle's restatement of
assemble_conduction (src/fem/thermal.cpp:92-141, pinned to the reference), for every
element family: conductivity matrix within 1e-12 relative Frobenius at the oracle's
entries (the extra topological entries zero to rounding), rhs (flux minus the eliminated prescribed temperatures) within 1e-12; and a
steady solve that reproduces the exact linear temperature profile between two faces."""
import ctypes as C

import numpy as np
import pytest
import torch
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from calculixpp_b200 import Plan, ThermalPlan
from calculixpp_b200 import meshgen as mg
from tests.helpers import ALL_TYPES, box_model, rel_fro, to_np

pytestmark = pytest.mark.gpu


def hot_cold(m, length):
    hot, cold = mg.face_nodes(m, 0, 0.0), mg.face_nodes(m, 0, float(length))
    return np.concatenate([hot, cold]), np.concatenate([np.full(hot.size, 100.0), np.full(cold.size, 20.0)])


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_conduction_matches_oracle(cuda, port, etype):
    quad = etype in (mg.C3D20, mg.C3D20R, mg.C3D15, mg.C3D10)
    dims = (2, 2, 2) if quad else (4, 3, 2)
    m = box_model(etype, *dims, jitter=0.08, seed=etype).mesh
    rng = np.random.default_rng(etype)
    k = rng.uniform(10.0, 60.0, m.n_elems)
    q = rng.uniform(-1.0, 1.0, m.n_nodes)
    tn, tv = hot_cold(m, dims[0])
    plan = ThermalPlan(m, tn, tv)
    vals, rhs = (to_np(t) for t in plan.assemble_conduction(k, q))
    deq, pre, nf = mg.thermal_dof_map(m.n_nodes, tn, tv)
    rp, ci, v, r = port.assemble_conduction(m, k, deq, pre, nf, q)
    rpg, cig = (to_np(t) for t in plan.pattern())
    # the reference omits exact-zero entries (frequent on the right-angled Kuhn tetrahedra);
    # the topological pattern holds them, to rounding zero
    kg = np.repeat(np.arange(nf), np.diff(rpg)).astype(np.int64) * nf + cig
    ko = np.repeat(np.arange(nf), np.diff(rp)).astype(np.int64) * nf + ci
    keep = np.isin(kg, ko)
    assert keep.sum() == ko.size
    assert rel_fro(vals[keep], v) <= 1e-12
    assert np.abs(vals[~keep]).max(initial=0.0) <= 1e-12 * np.abs(v).max()
    assert rel_fro(rhs, r) <= 1e-12
    plan.close()


def test_steady_linear_profile_and_plan_kind(cuda):
    m = box_model(mg.C3D10, 4, 2, 2, jitter=0.0, seed=0).mesh
    tn, tv = hot_cold(m, 4)
    plan = ThermalPlan(m, tn, tv)
    vals, rhs = plan.assemble_conduction(np.full(m.n_elems, 45.0))
    rp, ci = (to_np(t) for t in plan.pattern())
    A = sp.csr_matrix((to_np(vals), ci, rp), shape=(plan.n_free, plan.n_free))
    T = spla.spsolve(A.tocsc(), to_np(rhs))
    free = plan.t_dof_eq >= 0
    exact = 100.0 - 80.0 * m.coords[free, 0] / 4.0
    assert np.abs(T - exact).max() <= 1e-9 * 100.0
    plan.close()
    # a mechanical plan is rejected by the conduction entry point
    mech = Plan(box_model(mg.C3D8, 2, 1, 1))
    k = torch.full((2,), 45.0, dtype=torch.float64, device=mech.device)
    v = torch.empty(mech.nnz, dtype=torch.float64, device=mech.device)
    rc = mech.lib.cxg_assemble_conduction(mech.h, C.c_void_p(k.data_ptr()), None, C.c_void_p(v.data_ptr()), None,
                                          None)
    assert rc == 1 and b"cxg_thermal_plan_create" in mech.lib.cxg_last_error()


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_conduction_films_match_oracle(cuda, port, etype):
    """*FILM faces (thermal.cpp:113-126) against the oracle's restatement (pinned bit-exact
    to the reference): films on random faces, two on some elements, with prescribed
    temperatures on one face; matrix and rhs within 1e-12; clearing the films restores
    the film-free system."""
    from tests.test_oracle_thermal import film_case
    model, m, films, tn, tv = film_case(etype, 90 + etype)
    k = np.random.default_rng(etype).uniform(10.0, 60.0, m.n_elems)
    q = np.random.default_rng(etype + 1).uniform(-1.0, 1.0, m.n_nodes)
    plan = ThermalPlan(m, tn, tv)
    v0, r0 = (to_np(t).copy() for t in plan.assemble_conduction(k, q))
    plan.set_films(*films)
    vals, rhs = (to_np(t).copy() for t in plan.assemble_conduction(k, q))
    deq, pre, nf = mg.thermal_dof_map(m.n_nodes, tn, tv)
    rp, ci, v, r = port.assemble_conduction_films(m, k, deq, pre, nf, films, q)
    rpg, cig = (to_np(t) for t in plan.pattern())
    kg = np.repeat(np.arange(nf), np.diff(rpg)).astype(np.int64) * nf + cig
    ko = np.repeat(np.arange(nf), np.diff(rp)).astype(np.int64) * nf + ci
    keep = np.isin(kg, ko)
    assert keep.sum() == ko.size
    assert rel_fro(vals[keep], v) <= 1e-12
    assert np.abs(vals[~keep]).max(initial=0.0) <= 1e-12 * np.abs(v).max()
    assert rel_fro(rhs, r) <= 1e-12
    plan.set_films()
    v1, r1 = (to_np(t) for t in plan.assemble_conduction(k, q))
    assert np.array_equal(v1, v0) and np.array_equal(r1, r0)
    with pytest.raises(Exception):
        plan.set_films([0], [99], [1.0], [0.0])  # face out of range
    plan.close()
