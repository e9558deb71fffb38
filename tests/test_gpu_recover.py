"""Field recovery through the CUDA path: Gauss-point stress and nodal strain / stress /
reaction (recover_gauss_stress, recover_fields, src/fem/stress.cpp:147-271) against the
oracle's restatement (pinned to the reference), and equilibrium after a solve.

Bars: 1e-12 relative Frobenius for strains and stresses; reactions 1e-11 relative
(f_int is formed from the Gauss-point stresses here and as K_e u_e in the reference,
which agree to rounding)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from calculixpp_b200 import CxgError, Plan
from calculixpp_b200 import meshgen as mg
from tests.helpers import ALL_TYPES, box_model, rel_fro, to_np

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_recovery_matches_oracle(cuda, port, etype):
    quad = etype in (mg.C3D20, mg.C3D20R, mg.C3D15)
    dims = (2, 2, 2) if quad else (4, 3, 2)
    model = box_model(etype, *dims, jitter=0.08, seed=etype)
    m = model.mesh
    m.young = m.young * np.random.default_rng(etype).uniform(0.5, 1.5, m.n_elems)
    u = np.random.default_rng(etype + 3).uniform(-1e-3, 1e-3, 3 * m.n_nodes)
    plan = Plan(model)
    gs = to_np(plan.recover_gauss_stress(u))
    assert rel_fro(gs, port.recover_gauss_stress(m, m.young, m.poisson, u)) <= 1e-12
    f = model.external_load_vector()
    if etype == mg.C3D8R:
        with pytest.raises(CxgError) as exc:
            plan.recover_fields(u, f)
        assert exc.value.code == 5
        return
    st, ss, rf = (to_np(t) for t in plan.recover_fields(u, f))
    st0, ss0, rf0 = port.recover_fields(m, m.young, m.poisson, u, f)
    assert rel_fro(st, st0) <= 1e-12
    assert rel_fro(ss, ss0) <= 1e-12
    assert rel_fro(rf, rf0) <= 1e-11


def test_reactions_balance_the_load(cuda):
    model = box_model(mg.C3D20, 4, 2, 2, jitter=0.05, seed=9)
    plan = Plan(model)
    f = model.external_load_vector()
    vals, rhs = plan.assemble_linear(f)
    rp, ci = (to_np(t) for t in plan.pattern())
    A = sp.csr_matrix((to_np(vals), ci, rp), shape=(plan.n_free, plan.n_free))
    x = spla.spsolve(A.tocsc(), to_np(rhs))
    u = model.dof_map()[1].copy()
    free = model.dof_map()[0] >= 0
    u[free] = x
    _, _, rf = (to_np(t) for t in plan.recover_fields(u, f))
    rf = rf.reshape(-1)
    scale = np.abs(f).sum()
    assert np.abs(rf[free]).max() <= 1e-9 * scale        # equilibrium at free DOFs
    total = rf.reshape(-1, 3).sum(0) + f.reshape(-1, 3).sum(0)  # reactions carry the load
    assert np.abs(total).max() <= 1e-9 * scale
