"""solve_sparse (cxg_solve_sparse): ComputeBackend::solve_sparse on the device.

The reference's CPU backend (src/compute/cpu_backend.cpp:24-72) sums duplicate COO
triplets, then runs a sparse direct solve or IC0-preconditioned CG and throws when CG
misses its tolerance. The device kinds are held to a host direct solve of the same
system: direct within 1e-10, both CG kinds within 1e-8 at rtol 1e-10; the IC0 kind
needs fewer iterations than the diagonal one; an indefinite matrix and an iteration cap
end in CXG_ERR_NOT_CONVERGED with the reason.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from calculixpp_b200 import CxgError, Plan, solve_sparse
from calculixpp_b200 import meshgen as mg
from tests.helpers import box_model, rel_fro, to_np

pytestmark = pytest.mark.gpu


def _system(etype, dims, seed):
    """K_ff and rhs of a clamped, loaded, jittered box, as COO with a third of the entries
    split into two triplets each."""
    model = box_model(etype, *dims, jitter=0.1, seed=seed, young=mg.lognormal_young(
        mg.box_mesh(etype, *dims).n_elems, seed=seed))
    plan = Plan(model)
    vals, rhs = plan.assemble_linear(model.external_load_vector())
    rp, ci = (to_np(t) for t in plan.pattern())
    v, b = to_np(vals), to_np(rhs)
    n = b.size
    rows = np.repeat(np.arange(n), np.diff(rp))
    split = np.arange(0, v.size, 3)
    v2 = v.copy()
    half = 0.5 * v2[split]
    v2[split] -= half
    rows2 = np.concatenate([rows, rows[split]])
    cols2 = np.concatenate([ci, ci[split]])
    vals2 = np.concatenate([v2, half])
    A = sp.csr_matrix((v, ci, rp), shape=(n, n))
    return rows2, cols2, vals2, n, b, A


@pytest.mark.parametrize("etype,dims", [(mg.C3D8, (10, 4, 4)), (mg.C3D20, (5, 2, 2)), (mg.C3D10, (4, 3, 3))])
def test_solver_kinds_agree(cuda, etype, dims):
    rows, cols, vals, n, b, A = _system(etype, dims, seed=etype)
    want = spla.spsolve(A.tocsc(), b)
    x, it, _ = solve_sparse(rows, cols, vals, n, b, "direct")
    assert it == 0 and rel_fro(x, want) <= 1e-10
    x_ic, it_ic, rel_ic = solve_sparse(rows, cols, vals, n, b, "cg", rtol=1e-10)
    assert rel_ic <= 1e-10 and rel_fro(x_ic, want) <= 1e-8
    x_j, it_j, rel_j = solve_sparse(rows, cols, vals, n, b, "cg_jacobi", rtol=1e-10)
    assert rel_j <= 1e-10 and rel_fro(x_j, want) <= 1e-8
    assert 0 < it_ic < it_j, (it_ic, it_j)


def test_ic0_breakdown_and_iteration_cap(cuda):
    rows, cols, vals, n, b, A = _system(mg.C3D8, (6, 3, 3), seed=1)
    with pytest.raises(CxgError) as exc:
        solve_sparse(rows, cols, vals, n, b, "cg", rtol=1e-12, max_iter=2)
    assert exc.value.code == 8 and "did not converge" in str(exc.value)
    # a negative diagonal entry: no positive shift of the diagonal rescues the factor
    neg = vals.copy()
    d0 = np.flatnonzero((rows == 0) & (cols == 0))
    neg[d0] = -np.abs(neg[d0])
    with pytest.raises(CxgError) as exc:
        solve_sparse(rows, cols, neg, n, b, "cg")
    assert exc.value.code == 8 and "IC0" in str(exc.value)
