"""Material-point (J2) tangent assembly parity against the oracle's
assemble_material_tangent, over several increments with commits in between.

Bars (FP64): tangent values 1e-12 relative Frobenius, f_int 1e-12 relative, J2
history (plastic strain, equivalent plastic strain) within 1e-10 per Gauss point."""
import numpy as np
import pytest

from calculixpp_b200 import Plan
from calculixpp_b200 import meshgen as mg
from calculixpp_b200.assembly import Material
from tests.helpers import ALL_TYPES, box_model, per_element_materials, rel_fro, to_np

pytestmark = pytest.mark.gpu

J2_STEEL = Material(210000.0, 0.3, ([0.0, 1.0], [250.0, 1250.0]), 0)  # sy=250, H=1000


def displacement_field(model, strain, seed=0):
    """Bending-plus-stretch field: yields part of the body (ep > 0 on some points only)."""
    x = model.mesh.coords
    L = x.max(axis=0)
    rng = np.random.default_rng(seed)
    u = np.zeros_like(x)
    u[:, 0] = strain * x[:, 0] * (0.3 + x[:, 2] / L[2])
    u[:, 2] = -0.5 * strain * x[:, 0] ** 2 / L[0]
    u += rng.uniform(-1e-4, 1e-4, size=u.shape) * strain * L.max()
    return u.reshape(-1)


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_tangent_increments(cuda, port, etype):
    quad = etype in (mg.C3D20, mg.C3D20R, mg.C3D15)
    dims = (2, 2, 1) if quad else (4, 2, 2)
    model = box_model(etype, *dims, jitter=0.08, seed=etype, materials=[J2_STEEL], load=False)
    plan = Plan(model)
    mats, em = per_element_materials(model)
    dof_eq, pre, nf = model.dof_map()
    committed = np.zeros(plan.n_gauss * 13)
    yielded = 0.0
    for k in range(1, 4):
        u = displacement_field(model, 0.0006 * k, seed=k)
        vg, fg, rg = plan.assemble_tangent(u)
        rp, ci, v, rhs, fo, so = port.assemble_tangent(model.mesh, mats, em, dof_eq, pre, nf, u, committed)
        rpg, cig = (to_np(t) for t in plan.pattern())
        if np.array_equal(rpg, rp) and np.array_equal(cig, ci):
            assert rel_fro(to_np(vg), v) <= 1e-12, k
        else:  # topological pattern may carry exact-zero entries the oracle skips
            rows_g = np.repeat(np.arange(nf), np.diff(rpg)).astype(np.int64) * nf + cig
            rows_o = np.repeat(np.arange(nf), np.diff(rp)).astype(np.int64) * nf + ci
            keep = np.isin(rows_g, rows_o)
            assert rel_fro(to_np(vg)[keep], v) <= 1e-12, k
        assert rel_fro(to_np(fg), fo) <= 1e-12, k
        sg = to_np(plan.state(committed=False)).reshape(-1)
        scale = np.maximum(1.0, np.abs(so))
        assert np.all(np.abs(sg - so) <= 1e-10 * scale), k
        plan.commit()
        committed = so
        yielded = np.mean(so.reshape(-1, 13)[:, 6] > 0)
    assert 0.0 < yielded < 1.0, f"expected partial yielding, got {yielded:.2f}"


def test_commit_semantics(cuda):
    """Assembly writes only the trial history; commit promotes it (material_model.hpp:58-63)."""
    model = box_model(mg.C3D8, 3, 2, 2, materials=[J2_STEEL], load=False)
    plan = Plan(model)
    u = displacement_field(model, 0.006)
    plan.assemble_tangent(u)
    assert float(plan.state(committed=True)[:, 6].abs().max()) == 0.0
    trial = plan.state(committed=False).clone()
    assert float(trial[:, 6].max()) > 0.0
    plan.commit()
    assert bool((plan.state(committed=True) == trial).all())


def test_elastic_tangent_matches_linear(cuda):
    """Linear elasticity through the material-point path: same K as the linear
    assembly and f_int = K_full u (tests/test_element.cpp:106-135 at mesh level)."""
    model = box_model(mg.C3D20, 2, 2, 2, seed=4, load=False)
    plan = Plan(model)
    vl, _ = plan.assemble_linear()
    u = np.random.default_rng(0).uniform(-1e-3, 1e-3, 3 * model.mesh.n_nodes)
    dof_eq = model.dof_map()[0]
    u[dof_eq < 0] = 0.0
    vt, fi, _ = plan.assemble_tangent(u)
    assert rel_fro(to_np(vt), to_np(vl)) <= 1e-13
    import scipy.sparse as sp
    rp, ci = (to_np(t) for t in plan.pattern())
    K = sp.csr_matrix((to_np(vl), ci, rp), shape=(plan.n_free, plan.n_free))
    free = dof_eq >= 0
    ku = K @ u[free]
    assert np.abs(to_np(fi)[free] - ku).max() <= 1e-9 * np.abs(ku).max()


def test_state_roundtrip(cuda):
    model = box_model(mg.C3D6, 2, 2, 1, materials=[J2_STEEL], load=False)
    plan = Plan(model)
    s = np.random.default_rng(1).standard_normal((plan.n_gauss, 13))
    plan.set_state(s, committed=True)
    assert np.array_equal(to_np(plan.state(committed=True)), s)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("etype", ALL_TYPES)
def test_launch_shapes_give_identical_bits(cuda, etype, precision):
    """Every node-pair tile and grid shape of the element pass, and every row-gather
    block size, produce the same bits in the tangent and in the linear assembly."""
    quad = etype in (mg.C3D20, mg.C3D20R, mg.C3D15)
    model = box_model(etype, *((2, 2, 2) if quad else (4, 3, 2)), jitter=0.08, seed=etype, materials=[J2_STEEL],
                      load=False)
    plan = Plan(model, precision)
    u = displacement_field(model, 0.0012)
    ref_t = [t.clone() for t in plan.assemble_tangent(u)]
    ref_l = [t.clone() for t in plan.assemble_linear()]
    tiles = (0, 1, 2) if precision == "mixed" else (0, 1)
    for tile in tiles:
        for bps, warps in ((0, 0), (1, 2), (2, 8)):
            plan.set_launch_config(tangent=False, tile=tile, p1_blocks_per_sm=bps, p2_warps=warps)
            assert all(bool((a == b).all()) for a, b in zip(plan.assemble_linear(), ref_l)), (tile, bps, warps)
            if tile < 2:
                plan.set_launch_config(tangent=True, tile=tile, p1_blocks_per_sm=bps, p2_warps=warps)
                assert all(bool((a == b).all()) for a, b in zip(plan.assemble_tangent(u), ref_t)), (tile, bps, warps)
    with pytest.raises(Exception):
        plan.set_launch_config(tangent=True, tile=2)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_plan_tune_keeps_a_shape_and_the_bits(cuda, precision):
    """Plan.tune times the element-pass shapes, then the row gather's block sizes at the
    kept shape; what it keeps is one of those shapes, and the assembly through it (linear
    and tangent) is bit-identical to the default shape's."""
    model = box_model(mg.C3D20, 3, 2, 2, jitter=0.08, seed=3, materials=[J2_STEEL], load=False)
    plan = Plan(model, precision)
    u = displacement_field(model, 0.0012)
    ref_l = [t.clone() for t in plan.assemble_linear()]
    ref_t = [t.clone() for t in plan.assemble_tangent(u)]
    for tangent, step in ((False, lambda: plan.assemble_linear(check=False)), (True, lambda: plan.assemble_tangent(u))):
        shape = plan.tune(step, tangent=tangent, reps=2)
        assert shape["tile"] in (("2x4", "2x2") if tangent else ("2x4", "2x2", "4x4"))
        assert shape["p1_blocks_per_sm"] in (0, 1, 2) and shape["p2_warps"] in (2, 4, 8) and shape["ms"] > 0
    assert all(bool((a == b).all()) for a, b in zip(plan.assemble_linear(), ref_l))
    assert all(bool((a == b).all()) for a, b in zip(plan.assemble_tangent(u), ref_t))
