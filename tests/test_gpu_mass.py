"""Mass (consistent and lumped) and geometric-stiffness assembly through the CUDA path
against the oracle's restatement of assemble_mass / assemble_geometric_stiffness
(src/fem/assembly.cpp:259-331), for every element family.

Bar: values at the oracle's entries within 1e-12 relative Frobenius; entries of the
topological pattern that the reference omits as exact zeros (every off-diagonal entry of
the lumped mass) must be exactly 0.0."""
import numpy as np
import pytest

from calculixpp_b200 import Plan
from calculixpp_b200 import meshgen as mg
from tests.helpers import ALL_TYPES, box_model, rel_fro, to_np

pytestmark = pytest.mark.gpu


def compare(plan, nf, vg, rp, ci, v):
    rpg, cig = (to_np(t) for t in plan.pattern())
    kg = np.repeat(np.arange(nf), np.diff(rpg)).astype(np.int64) * nf + cig
    ko = np.repeat(np.arange(nf), np.diff(rp)).astype(np.int64) * nf + ci
    keep = np.isin(kg, ko)
    assert keep.sum() == ko.size
    assert rel_fro(vg[keep], v) <= 1e-12
    assert np.all(vg[~keep] == 0.0)


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_mass_and_geometric_match_oracle(cuda, port, etype):
    quad = etype in (mg.C3D20, mg.C3D20R, mg.C3D15)
    dims = (2, 2, 2) if quad else (4, 3, 2)
    model = box_model(etype, *dims, jitter=0.08, seed=etype, prescribe=0.01)
    m = model.mesh
    rng = np.random.default_rng(etype)
    rho = rng.uniform(2.7e-9, 7.9e-9, m.n_elems)
    gs = rng.normal(0.0, 80.0, (m.n_elems * mg.NGP[etype], 6))
    dof_eq, pre, nf = model.dof_map()
    plan = Plan(model, "mixed")  # the operators run in FP64 whatever the plan's precision
    for kind in ("mass", "lumped", "geometric"):
        if kind == "geometric":
            vg = to_np(plan.assemble_geometric_stiffness(gs))
        else:
            vg = to_np(plan.assemble_mass(rho, lumped=kind == "lumped"))
        rp, ci, v = port.assemble_scalar(kind, m, dof_eq, pre, nf, density=rho, gp_stress=gs)
        compare(plan, nf, vg, rp, ci, v)
    # the linear stiffness still assembles correctly after the FP64 buffer was used
    vl, _ = plan.assemble_linear()
    assert np.isfinite(to_np(vl)).all()
    plan.close()


def test_mass_total_and_zero_stress(cuda):
    """Total translational mass: sum of M over one direction's DOFs equals rho V for an
    unconstrained body; a zero stress field gives a zero K_geo."""
    model = box_model(mg.C3D20, 3, 2, 2, jitter=0.05, seed=1, load=False)
    model.spc = None
    plan = Plan(model)
    m = model.mesh
    rho = np.full(m.n_elems, 7.85e-9)
    M = to_np(plan.assemble_mass(rho))
    rp, ci = (to_np(t) for t in plan.pattern())
    rows = np.repeat(np.arange(plan.n_free), np.diff(rp))
    x_dir = (rows % 3 == 0) & (ci % 3 == 0)
    volume = 3.0 * 2.0 * 2.0
    assert abs(M[x_dir].sum() - 7.85e-9 * volume) <= 1e-12 * 7.85e-9 * volume
    Ml = to_np(plan.assemble_mass(rho, lumped=True))
    assert abs(Ml.sum() - 3 * 7.85e-9 * volume) <= 1e-12 * 3 * 7.85e-9 * volume
    assert not np.any(to_np(plan.assemble_geometric_stiffness(None)))
