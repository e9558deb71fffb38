"""Element-level parity of the CUDA kernels against the oracle (the C restatement of
element_stiffness / element_tangent_force / J2PlasticMaterial::evaluate).

Tolerances: FP64 path 1e-12 relative Frobenius on K_e and f_e, 1e-10 on the J2
history per Gauss point; mixed path (FP32 gradients and Gram blocks) 2e-5 relative on
K_e."""
import numpy as np
import pytest

from calculixpp_b200 import CxgError, Material, element_stiffness, element_tangent_force
from calculixpp_b200 import meshgen as mg
from tests.helpers import ALL_TYPES, ISO_TABLE, distorted_elements, rel_fro, to_np, unit_element

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 2e-5
STATE_TOL = 1e-10


@pytest.mark.parametrize("etype", ALL_TYPES)
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_element_stiffness(cuda, port, etype, precision):
    B = 48
    X = distorted_elements(etype, B, seed=etype)
    E = np.linspace(70e3, 210e3, B)
    nu = np.linspace(0.25, 0.35, B)
    K = to_np(element_stiffness(etype, X, E, nu, precision=precision))
    tol = FP64_TOL if precision == "fp64" else MIXED_TOL
    worst = 0.0
    for b in range(B):
        Ko = port.element_stiffness(etype, X[b], E[b], nu[b])
        worst = max(worst, rel_fro(K[b], Ko))
    assert worst <= tol, f"{mg.NAMES[etype]} {precision}: rel Frobenius {worst:.3e}"


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_element_stiffness_unit_symmetric(cuda, port, etype):
    x = unit_element(etype)
    K = to_np(element_stiffness(etype, x, 210000.0, 0.3))
    assert np.array_equal(K, K.T)
    assert rel_fro(K, port.element_stiffness(etype, x, 210000.0, 0.3)) <= FP64_TOL


def _plastic_cases(etype, seed):
    rng = np.random.default_rng(100 + seed)
    X = distorted_elements(etype, 16, seed=seed)
    n = mg.NODES[etype]
    # linear displacement field with ~1% strain plus noise: well past yield (800/210000)
    U = np.empty_like(X)
    for b in range(X.shape[0]):
        G = rng.uniform(-0.012, 0.012, size=(3, 3))
        U[b] = X[b] @ G.T + rng.uniform(-1e-3, 1e-3, size=(n, 3))
    return X, U


MATERIALS = {
    "elastic": Material(210000.0, 0.3),
    "iso": Material(210000.0, 0.3, ISO_TABLE, 0),
    "kinematic": Material(210000.0, 0.3, ISO_TABLE, 1),
    "combined": Material(210000.0, 0.3, ISO_TABLE, 2, 5000.0),
    "perfect": Material(210000.0, 0.3, ([0.0], [800.0]), 0),
    "multilinear": Material(200000.0, 0.29, ([0.0, 0.01, 0.03, 0.1], [300.0, 420.0, 500.0, 520.0]), 0),
}


@pytest.mark.parametrize("etype", ALL_TYPES)
@pytest.mark.parametrize("mname", list(MATERIALS))
def test_element_tangent_force(cuda, port, etype, mname):
    from oracle.oracle import make_material
    mat = MATERIALS[mname]
    om = make_material(mat.E, mat.nu, mat.plastic, mat.hardening, mat.h_kin)
    X, U = _plastic_cases(etype, etype)
    ngp = mg.NGP[etype]
    # two steps: from a virgin history, then from the committed trial history of step 1
    committed = np.zeros((X.shape[0], ngp, 13))
    for step in range(2):
        Uk = U * (step + 1) / 2.0
        Kg, fg, sg = (to_np(t) for t in element_tangent_force(etype, X, Uk, mat, committed))
        for b in range(X.shape[0]):
            Ko, fo, so = port.element_tangent_force(etype, X[b], Uk[b], om, committed[b].ravel())
            assert rel_fro(Kg[b], Ko) <= FP64_TOL, (mname, step, b, rel_fro(Kg[b], Ko))
            assert rel_fro(fg[b], fo) <= FP64_TOL, (mname, step, b, rel_fro(fg[b], fo))
            scale = np.maximum(1.0, np.abs(so))
            assert np.all(np.abs(sg[b] - so) <= STATE_TOL * scale), (mname, step, b)
        committed = sg
    if mat.plastic is not None:
        assert np.any(committed[:, :, 6] > 0.0), "cases must reach the plastic branch"


def test_material_point_equals_stiffness_at_zero(cuda):
    """element_tangent_force at u = 0 reproduces element_stiffness (tests/test_element.cpp:106-135)."""
    for etype in ALL_TYPES:
        X = distorted_elements(etype, 8, seed=3)
        K0 = to_np(element_stiffness(etype, X, 210000.0, 0.3))
        Kt, fe, _ = (to_np(t) for t in element_tangent_force(etype, X, np.zeros_like(X), MATERIALS["elastic"]))
        assert rel_fro(Kt, K0) <= 1e-14
        assert np.abs(fe).max() <= 1e-9


def test_internal_force_is_K_times_u(cuda):
    """fe = Ke ue for linear elasticity (tests/test_element.cpp:124-134)."""
    for etype in ALL_TYPES:
        X = distorted_elements(etype, 8, seed=4)
        U = np.random.default_rng(etype).uniform(-1e-3, 1e-3, X.shape)
        K = to_np(element_stiffness(etype, X, 210000.0, 0.3))
        _, fe, _ = (to_np(t) for t in element_tangent_force(etype, X, U, MATERIALS["elastic"]))
        ku = np.einsum("bij,bj->bi", K, U.reshape(U.shape[0], -1))
        assert np.abs(fe - ku).max() <= 1e-7 * (1.0 + np.abs(ku).max())


def test_negative_jacobian_reported(cuda):
    """An inverted element raises the reference's message (src/fem/element.cpp:86-88)."""
    x = unit_element(mg.C3D8)
    bad = x[[4, 5, 6, 7, 0, 1, 2, 3]]  # top and bottom swapped: det J < 0
    X = np.stack([x, bad, x])
    with pytest.raises(CxgError) as exc:
        element_stiffness(mg.C3D8, X, 210000.0, 0.3)
    assert exc.value.code == 4
    assert "non-positive element Jacobian" in str(exc.value)
    assert "index 1" in str(exc.value)
