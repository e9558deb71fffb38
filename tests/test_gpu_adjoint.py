"""Adjoint of the compliance and the device solve.

* dc/dX of the 4x2x2 C3D8 cantilever against the reference's own solve_sensitivity
  output (tests/golden, semi-analytic central differences with h = 1e-4): 1e-6 relative.
* dc/dE and dc/dX against central finite differences (step 1e-6, 64 random components)
  through the differentiable forward (device assembly + device CG at rtol 1e-12); the
  dc/dX bar adds the difference quotient's CG noise, about rtol*|c|/h.
* every full-integration family: dc/dX against the oracle's per-element central
  differences of K_e.
* the device CG against scipy's direct solve; non-convergence reported as an error."""
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

from calculixpp_b200 import CxgError, Plan
from calculixpp_b200 import meshgen as mg
from calculixpp_b200.adjoint import compliance
from tests.helpers import box_model, rel_fro, to_np

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_vectors.npz"))


def host_solution(plan, f):
    vals, rhs = plan.assemble_linear(f)
    rp, ci = (to_np(t) for t in plan.pattern())
    A = sp.csr_matrix((to_np(vals), ci, rp), shape=(plan.n_free, plan.n_free))
    x = spla.spsolve(A.tocsc(), to_np(rhs))
    return x, to_np(rhs)


def test_dcdX_matches_reference_sensitivity(cuda):
    model = box_model(mg.C3D8, 4, 2, 2, jitter=0.05, seed=5)
    assert np.array_equal(model.mesh.coords, GOLD["sens_coords"])
    plan = Plan(model)
    f = model.external_load_vector()
    x, rhs = host_solution(plan, f)
    assert abs(x @ rhs - float(GOLD["sens_compliance"])) <= 1e-9 * abs(x @ rhs)
    u = to_np(plan.expand(torch.as_tensor(x, device=plan.device)))
    _, dX = plan.adjoint_compliance(u)
    gold = GOLD["sens_dcdX"]
    assert np.abs(to_np(dX) - gold).max() <= 1e-6 * np.abs(gold).max()


def cantilever_rho(nx=6, ny=3, nz=3, seed=0):
    model = box_model(mg.C3D8, nx, ny, nz, jitter=0.05, seed=seed)
    rho = np.random.default_rng(seed).uniform(0.1, 1.0, model.mesh.n_elems)
    model.mesh.young = 210000.0 * rho ** 3
    return model


def test_autograd_matches_central_differences(cuda):
    model = cantilever_rho()
    plan = Plan(model)
    f = model.external_load_vector()
    dev = plan.device
    E = torch.as_tensor(model.mesh.young, device=dev).requires_grad_(True)
    X = torch.as_tensor(model.mesh.coords, device=dev).requires_grad_(True)
    c = compliance(E, X, plan, f)
    x, rhs = host_solution(plan, f)
    assert abs(float(c) - x @ rhs) <= 1e-10 * abs(x @ rhs)
    gE, gX = torch.autograd.grad(c, (E, X))
    rng = np.random.default_rng(1)
    free_nodes = np.nonzero(model.dof_map()[0].reshape(-1, 3)[:, 0] >= 0)[0]

    def c_at(Ev, Xv):
        with torch.no_grad():
            return float(compliance(Ev, Xv, plan, f))

    for k in rng.choice(model.mesh.n_elems, 32, replace=False):
        h = 1e-6 * float(E[k])
        Ep, Em = E.detach().clone(), E.detach().clone()
        Ep[k] += h
        Em[k] -= h
        fd = (c_at(Ep, X.detach()) - c_at(Em, X.detach())) / (2 * h)
        assert abs(fd - float(gE[k])) <= 1e-5 * abs(float(gE[k])) + 1e-12 * abs(float(c)), (k, fd, float(gE[k]))
    # each compliance evaluation carries the CG's own error (the forward's CG stops at
    # rtol 1e-12, about rtol*|c|); the two evaluations of a central difference take
    # different CG paths, so the quotient carries up to ~rtol*|c|/h of noise on top of
    # the 1e-5 relative bar
    cg_noise = 4 * 1e-12 * abs(float(c))
    for k in range(32):
        node = int(rng.choice(free_nodes))
        comp = int(rng.integers(3))
        h = 1e-6
        Xp, Xm = X.detach().clone(), X.detach().clone()
        Xp[node, comp] += h
        Xm[node, comp] -= h
        fd = (c_at(E.detach(), Xp) - c_at(E.detach(), Xm)) / (2 * h)
        g = float(gX[node, comp])
        tol = 1e-5 * max(abs(g), 1e-3 * float(gX.abs().max())) + cg_noise / h
        assert abs(fd - g) <= tol, (node, comp, fd, g, tol)


@pytest.mark.parametrize("etype", [mg.C3D20, mg.C3D20R, mg.C3D6, mg.C3D15, mg.C3D4, mg.C3D10])
def test_dcdX_all_families_against_element_differences(cuda, port, etype):
    model = box_model(etype, 2, 2, 2, jitter=0.08, seed=etype)
    plan = Plan(model)
    f = model.external_load_vector()
    x, _ = host_solution(plan, f)
    u = to_np(plan.expand(torch.as_tensor(x, device=plan.device))).reshape(-1, 3)
    dE, dX = plan.adjoint_compliance(u.reshape(-1))
    m = model.mesh
    ref = np.zeros((m.n_nodes, 3))
    refE = np.zeros(m.n_elems)
    for e in range(m.n_elems):
        c = m.conn[e]
        ref[c] += port.element_compliance_grad_fd(etype, m.coords[c], u[c], m.young[e], 0.3, 1e-5)
        Ke = port.element_stiffness(etype, m.coords[c], m.young[e], 0.3)
        refE[e] = -(u[c].ravel() @ Ke @ u[c].ravel()) / m.young[e]
    assert np.abs(to_np(dX) - ref).max() <= 1e-6 * np.abs(ref).max()
    assert rel_fro(to_np(dE), refE) <= 1e-12


def test_device_cg_matches_direct_solve(cuda):
    cfg = mg.cantilever_c3d8_config1()
    from calculixpp_b200.assembly import Material, Model
    m, tip = cfg["mesh"], cfg["tip"]
    model = Model(m, [Material(210000.0, 0.3)], None, cfg["spc"],
                  (tip, np.full(tip.size, 2), np.full(tip.size, -1000.0 / tip.size)))
    plan = Plan(model)
    vals, rhs = plan.assemble_linear(model.external_load_vector())
    x, iters, rel = plan.solve_cg(vals, rhs, rtol=1e-13, max_iter=20000)
    xd, _ = host_solution(plan, model.external_load_vector())
    assert rel <= 1e-13 and iters > 0
    assert rel_fro(to_np(x), xd) <= 1e-9
    y = plan.spmv(vals, x)  # true residual; CG's recurrence residual drifts from it
    assert rel_fro(to_np(y), to_np(rhs)) <= 1e-9
    with pytest.raises(CxgError) as exc:
        plan.solve_cg(vals, rhs, rtol=1e-14, max_iter=5)
    assert exc.value.code == 8 and "did not converge" in str(exc.value)


def test_adjoint_rejects_reduced_hex(cuda):
    plan = Plan(box_model(mg.C3D8R, 2, 1, 1))
    with pytest.raises(CxgError) as exc:
        plan.adjoint_compliance(np.zeros(3 * plan.model.mesh.n_nodes))
    assert exc.value.code == 5


def test_adjoint_identities(cuda):
    """Size-independent checks of the adjoint, used at full size by the bench:
    K is linear in E, so sum_e E_e dc/dE_e = -c; a rigid translation of every node leaves
    c unchanged, so sum_nodes dc/dX = 0; K scales like the length in 3-D elasticity, so
    sum X . dc/dX = -c."""
    model = cantilever_rho(8, 4, 3, seed=3)
    plan = Plan(model)
    f = model.external_load_vector()
    x, rhs = host_solution(plan, f)
    c = float(x @ rhs)
    u = to_np(plan.expand(torch.as_tensor(x, device=plan.device)))
    dE, dX = (to_np(t) for t in plan.adjoint_compliance(u))
    X = model.mesh.coords
    assert abs(float(model.mesh.young @ dE) + c) <= 1e-10 * abs(c)
    assert np.abs(dX.reshape(-1, 3).sum(0)).max() <= 1e-9 * np.abs(dX).sum()
    assert abs(float((X.reshape(-1) * dX.reshape(-1)).sum()) + c) <= 1e-9 * abs(c)
