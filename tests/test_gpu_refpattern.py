"""cxg_plan_use_reference_pattern: the linear assembly on the reference's own CSR pattern.

The reference's scatter skips every element contribution that is exactly 0.0
(src/fem/assembly.cpp:86-90); on straight, axis-aligned elements (unit boxes) and on
tetrahedra with faces on the box boundary, some entries get nothing but exact zeros and
are absent from its LinearSystem. With the mode on, row_ptr and col_idx must equal the
oracle's (pinned bit-for-bit to the reference) exactly, for every family, on unit and
jittered boxes, and the values and rhs must match within 1e-12; the dropped entries
carried only rounding in the topological assembly; SpMV and CG use the same pattern;
switching the mode off restores the topological pattern.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from calculixpp_b200 import CxgError, Plan
from calculixpp_b200 import meshgen as mg
from tests.helpers import ALL_TYPES, box_model, per_element_materials, rel_fro, to_np

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("jitter", [0.0, 0.08])
@pytest.mark.parametrize("etype", ALL_TYPES)
def test_reference_pattern_equals_oracle(cuda, port, etype, jitter):
    quad = etype in (mg.C3D20, mg.C3D20R, mg.C3D15, mg.C3D10)
    dims = (3, 2, 2) if quad else (5, 3, 2)
    model = box_model(etype, *dims, jitter=jitter, seed=etype)
    m = model.mesh
    mats, em = per_element_materials(model)
    dof_eq, pre, nf = model.dof_map()
    f = model.external_load_vector()
    rp, ci, vo, rhs_o = port.assemble_linear(m, mats, em, dof_eq, pre, nf, f)
    plan = Plan(model)
    topo_nnz = plan.nnz
    v_topo = to_np(plan.assemble_linear(f)[0]).copy()
    rp_t, ci_t = (to_np(t).copy() for t in plan.pattern())
    plan.use_reference_pattern()
    assert plan.nnz == ci.size
    vg, rg = plan.assemble_linear(f)
    rpg, cig = (to_np(t) for t in plan.pattern())
    assert np.array_equal(rpg, rp)
    assert np.array_equal(cig, ci)
    assert rel_fro(to_np(vg), vo) <= 1e-12
    assert rel_fro(to_np(rg), rhs_o) <= 1e-12
    # the dropped entries carried only rounding in the topological assembly
    kt = np.repeat(np.arange(nf), np.diff(rp_t)).astype(np.int64) * nf + ci_t
    ko = np.repeat(np.arange(nf), np.diff(rp)).astype(np.int64) * nf + ci
    dropped = ~np.isin(kt, ko)
    assert dropped.sum() == topo_nnz - ci.size
    assert np.abs(v_topo[dropped]).max(initial=0.0) <= 1e-12 * np.abs(v_topo).max()
    # SpMV on the same pattern
    x = np.random.default_rng(etype).standard_normal(nf)
    A = sp.csr_matrix((vo, ci, rp), shape=(nf, nf))
    assert rel_fro(to_np(plan.spmv(vg, torch.as_tensor(x, device=plan.device))), A @ x) <= 1e-12
    plan.use_reference_pattern(False)
    assert plan.nnz == topo_nnz


def test_reference_pattern_drops_entries_on_unit_boxes(cuda):
    """The unit C3D20 / C3D20R / C3D6 / C3D15 boxes do have entries the reference leaves out."""
    for etype in (mg.C3D20, mg.C3D20R, mg.C3D6, mg.C3D15):
        dims = (3, 2, 2) if etype != mg.C3D6 else (5, 3, 2)
        plan = Plan(box_model(etype, *dims, jitter=0.0, seed=etype))
        topo = plan.nnz
        plan.use_reference_pattern()
        assert plan.nnz < topo, mg.TYPE_NAMES[etype]


def test_reference_pattern_limits(cuda):
    model = box_model(mg.C3D20, 2, 2, 1, jitter=0.0)
    plan = Plan(model)
    plan.use_reference_pattern()
    with pytest.raises(CxgError) as exc:
        plan.assemble_tangent(np.zeros(3 * model.mesh.n_nodes))
    assert exc.value.code == 5 and "reference pattern" in str(exc.value)
    with pytest.raises(CxgError):
        plan.accumulate_linear(torch.zeros(plan.nnz, dtype=torch.float64, device=plan.device))
    plan.use_reference_pattern(False)
    plan.assemble_tangent(np.zeros(3 * model.mesh.n_nodes))
