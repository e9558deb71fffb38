"""The reference's own known-answer tests for this path, run against the oracle.

Restated from tests/test_element.cpp (partition of unity 1e-12, gradient consistency
1e-10, volumes 1e-12, constant-strain patch 1e-11, symmetry + six rigid-body modes
1e-3, hourglass energy > 1, material point = element_stiffness 1e-12, fe = Ke ue 1e-7)
and tests/test_plasticity.cpp (elastic below yield 1e-9, return onto the yield
surface 1e-6/1e-5, consistent tangent vs central differences h = 1e-7 within
1e-3 (|D|+1), kinematic back stress, commit semantics)."""
import numpy as np
import pytest

from calculixpp_b200 import meshgen as mg
from oracle.oracle import make_material
from tests.helpers import ALL_TYPES, ISO_TABLE, unit_element

VOL = {mg.C3D8: 1.0, mg.C3D8R: 1.0, mg.C3D20: 1.0, mg.C3D20R: 1.0, mg.C3D6: 0.5, mg.C3D15: 0.5,
       mg.C3D4: 1.0 / 6.0, mg.C3D10: 1.0 / 6.0}  # unit cube, wedge half, Kuhn tetrahedron


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_partition_of_unity(port, etype):
    for xi, et, ze, _ in port.gauss_rule(etype):
        N, dN = port.shape(etype, xi, et, ze)
        assert abs(N.sum() - 1.0) <= 1e-12
        assert np.abs(dN.sum(axis=0)).max() <= 1e-12


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_gradient_consistency_and_volume(port, etype):
    x = unit_element(etype)
    for xi, et, ze, _ in port.gauss_rule(etype):
        g, det = port.physical_gradients(etype, xi, et, ze, x)
        assert det > 0
        assert np.abs(g.sum(axis=0)).max() <= 1e-10
        assert np.abs(g.T @ x - np.eye(3)).max() <= 1e-10
    assert abs(port.element_volume(etype, x) - VOL[etype]) <= 1e-12


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_constant_strain_patch(port, etype):
    x = unit_element(etype)
    exx, eyy, ezz, gxy, gxz, gyz = 1e-3, -4e-4, 2e-4, 6e-4, -3e-4, 5e-4
    S = np.array([[exx, 0.5 * gxy, 0.5 * gxz], [0.5 * gxy, eyy, 0.5 * gyz], [0.5 * gxz, 0.5 * gyz, ezz]])
    ue = x @ S.T
    for xi, et, ze, _ in port.gauss_rule(etype):
        g, _ = port.physical_gradients(etype, xi, et, ze, x)
        H = ue.T @ g  # H_ij = sum_k u_ki g_kj
        eps = [H[0, 0], H[1, 1], H[2, 2], H[0, 1] + H[1, 0], H[0, 2] + H[2, 0], H[1, 2] + H[2, 1]]
        assert np.allclose(eps, [exx, eyy, ezz, gxy, gxz, gyz], atol=1e-11, rtol=0)


def rigid_modes(x):
    out = []
    for m in range(6):
        d = np.zeros_like(x)
        if m < 3:
            d[:, m] = 1.0
        elif m == 3:
            d[:, 0], d[:, 1] = -x[:, 1], x[:, 0]
        elif m == 4:
            d[:, 0], d[:, 2] = -x[:, 2], x[:, 0]
        else:
            d[:, 1], d[:, 2] = -x[:, 2], x[:, 1]
        out.append(d.ravel())
    return out


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_symmetry_and_rigid_body_null_space(port, etype):
    x = unit_element(etype)
    K = port.element_stiffness(etype, x, 210000.0, 0.3)
    assert np.abs(K - K.T).max() <= 1e-6
    for v in rigid_modes(x):
        assert np.linalg.norm(K @ v) <= 1e-3


def test_hourglass_mode_suppressed(port):
    K = port.element_stiffness(mg.C3D8R, unit_element(mg.C3D8R), 210000.0, 0.3)
    u = np.zeros(24)
    u[0::3] = [1, 1, -1, -1, -1, -1, 1, 1]
    assert u @ K @ u > 1.0


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_material_point_kernel(port, etype):
    x = unit_element(etype)
    mat = make_material(210000.0, 0.3)
    K = port.element_stiffness(etype, x, 210000.0, 0.3)
    K0, f0, _ = port.element_tangent_force(etype, x, np.zeros_like(x), mat)
    assert np.all(np.abs(K0 - K) <= 1e-12 * (1.0 + np.abs(K)))
    assert np.abs(f0).max() <= 1e-9
    n = mg.NODES[etype]
    ue = np.array([[0.001 * (k + 1), -0.002 * k, 0.0007 * (k + 2)] for k in range(n)])
    _, f1, _ = port.element_tangent_force(etype, x, ue, mat)
    ku = K @ ue.ravel()
    assert np.all(np.abs(f1 - ku) <= 1e-7 * (1.0 + np.abs(ku)))


def von_mises(s):
    p = s[:3].sum() / 3.0
    d = s[:3] - p
    return np.sqrt(3.0 * (0.5 * (d @ d) + s[3] ** 2 + s[4] ** 2 + s[5] ** 2))


def test_elastic_below_yield(port):
    jp, el = make_material(210000.0, 0.3, ISO_TABLE), make_material(210000.0, 0.3)
    strain = np.array([1e-4, -3e-5, -3e-5, 2e-5, 0.0, 1e-5])
    s1, D1, st = port.material_evaluate(jp, strain)
    s2, D2, _ = port.material_evaluate(el, strain)
    assert np.allclose(s1, s2, atol=1e-9, rtol=0) and np.allclose(D1, D2, atol=1e-9, rtol=0)
    assert st[6] == 0.0


def test_return_to_yield_surface(port):
    strain = np.array([0.01, -0.003, -0.003, 0.0, 0.0, 0.0])
    s, _, st = port.material_evaluate(make_material(210000.0, 0.3, ([0.0], [800.0])), strain)
    assert abs(von_mises(s) - 800.0) <= 1e-6 and st[6] > 0
    s, _, st = port.material_evaluate(make_material(210000.0, 0.3, ISO_TABLE), strain)
    assert abs(von_mises(s) - (800.0 + 8000.0 * st[6])) <= 1e-5


@pytest.mark.parametrize("hardening,hkin", [(0, 0.0), (2, 5000.0)])
def test_consistent_tangent_fd(port, hardening, hkin):
    mat = make_material(210000.0, 0.3, ISO_TABLE, hardening, hkin)
    strain = np.array([0.008, -0.0015, -0.002, 0.0012, 0.0006, -0.0004])
    _, D, st = port.material_evaluate(mat, strain)
    assert st[6] > 0
    h = 1e-7
    for j in range(6):
        ep, em = strain.copy(), strain.copy()
        ep[j] += h
        em[j] -= h
        fd = (port.material_evaluate(mat, ep)[0] - port.material_evaluate(mat, em)[0]) / (2 * h)
        assert np.all(np.abs(fd - D[:, j]) <= 1e-3 * (np.abs(D[:, j]) + 1.0))


def test_kinematic_back_stress(port):
    mat = make_material(210000.0, 0.3, ISO_TABLE, 1)
    s, _, st = port.material_evaluate(mat, np.array([0.01, -0.003, -0.003, 0.0, 0.0, 0.0]))
    alpha = st[7:]
    assert np.abs(alpha).max() > 1e-6
    p = s[:3].sum() / 3.0
    xi = np.concatenate([s[:3] - p - alpha[:3], s[3:] - alpha[3:]])
    assert abs(von_mises(xi) - 800.0) <= 1e-4


def test_commit_semantics(port):
    mat = make_material(210000.0, 0.3, ISO_TABLE)
    strain = np.array([0.01, -0.003, -0.003, 0.0, 0.0, 0.0])
    _, _, trial = port.material_evaluate(mat, strain)
    assert trial[6] > 0
    _, _, trial2 = port.material_evaluate(mat, strain, trial)  # re-evaluate from committed trial
    assert trial2[6] >= trial[6] - 1e-12
