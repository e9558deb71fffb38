"""Assembly parity of the CUDA path against the oracle's assemble_linear_static.

Bars (FP64 path): CSR pattern (row_ptr, col_idx) bit-exact; values and rhs within
1e-12 relative Frobenius; nodal displacements within 1e-10 relative L2 after the same
sparse direct solve (scipy SuperLU on both operators). Mixed path: displacements within
1e-6 relative L2 of the FP64 oracle."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from calculixpp_b200 import Plan, assemble_linear_static
from calculixpp_b200 import meshgen as mg
from calculixpp_b200.assembly import Material, Model
from tests.helpers import ALL_TYPES, box_model, per_element_materials, rel_fro, to_np

pytestmark = pytest.mark.gpu


def oracle_system(port, model):
    mats, em = per_element_materials(model)
    dof_eq, pre, nf = model.dof_map()
    return port.assemble_linear(model.mesh, mats, em, dof_eq, pre, nf, model.external_load_vector())


def solve(n, rp, ci, v, rhs):
    A = sp.csr_matrix((v, ci, rp), shape=(n, n))
    return spla.spsolve(A.tocsc(), rhs)


def compare_patterns(rp_g, ci_g, v_g, rp_o, ci_o, v_o, n):
    """GPU pattern is topological; the oracle's skips exact-zero contributions. Equal
    where the oracle has every topological entry; otherwise the extra GPU entries are
    numerically zero and the shared ones agree."""
    if np.array_equal(rp_g, rp_o) and np.array_equal(ci_g, ci_o):
        return v_g, v_o, True
    rows_g = np.repeat(np.arange(n), np.diff(rp_g))
    rows_o = np.repeat(np.arange(n), np.diff(rp_o))
    kg = rows_g.astype(np.int64) * n + ci_g
    ko = rows_o.astype(np.int64) * n + ci_o
    assert np.all(np.isin(ko, kg)), "oracle entry missing from the GPU pattern"
    extra = ~np.isin(kg, ko)
    assert np.abs(v_g[extra]).max() <= 1e-12 * np.abs(v_g).max()
    return v_g[~extra], v_o, False


def test_config1_cantilever_pattern_values_displacement(cuda, port):
    cfg = mg.cantilever_c3d8_config1()
    m = cfg["mesh"]
    tip = cfg["tip"]
    model = Model(m, [Material(210000.0, 0.3)], None, cfg["spc"],
                  (tip, np.full(tip.size, 2), np.full(tip.size, -1000.0 / tip.size)))
    sysg = assemble_linear_static(model)
    rp, ci, v, rhs = oracle_system(port, model)
    assert sysg.n_free == 1500 and v.size == 88218
    assert np.array_equal(to_np(sysg.row_ptr), rp)
    assert np.array_equal(to_np(sysg.col_idx), ci)
    vg = to_np(sysg.vals)
    assert rel_fro(vg, v) <= 1e-12
    assert rel_fro(to_np(sysg.rhs), rhs) <= 1e-12
    ug = solve(1500, rp, ci, vg, to_np(sysg.rhs))
    uo = solve(1500, rp, ci, v, rhs)
    assert rel_fro(ug, uo) <= 1e-10
    # The cantilever is a plain-FP64 configuration. Its mixed-precision displacement is
    # held to 5e-6: the aspect-10 beam's element rotations are ~10x its strains, and the
    # FP32 Gram blocks keep the rotation null space only to FP32 rounding (the 1e-6
    # bar of the mixed path applies to the block workloads, tested below).
    plan = sysg.extra["plan"]
    plan.set_precision("mixed")
    vm, rm = plan.assemble_linear(model.external_load_vector())
    um = solve(1500, rp, ci, to_np(vm), to_np(rm))
    assert rel_fro(um, uo) <= 5e-6


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_all_families_small_box(cuda, port, etype):
    quad = etype in (mg.C3D20, mg.C3D20R, mg.C3D15)
    dims = (2, 2, 2) if quad else (3, 2, 2)
    E = np.random.default_rng(etype).uniform(70e3, 210e3, size=mg.box_mesh(etype, *dims).n_elems)
    model = box_model(etype, *dims, jitter=0.1, seed=etype, young=E)
    sysg = assemble_linear_static(model)
    rp, ci, v, rhs = oracle_system(port, model)
    vg_cmp, vo_cmp, exact = compare_patterns(to_np(sysg.row_ptr), to_np(sysg.col_idx), to_np(sysg.vals),
                                             rp, ci, v, sysg.n_free)
    assert rel_fro(vg_cmp, vo_cmp) <= 1e-12
    assert rel_fro(to_np(sysg.rhs), rhs) <= 1e-12
    ug = solve(sysg.n_free, to_np(sysg.row_ptr), to_np(sysg.col_idx), to_np(sysg.vals), to_np(sysg.rhs))
    uo = solve(sysg.n_free, rp, ci, v, rhs)
    assert rel_fro(ug, uo) <= 1e-10
    plan = sysg.extra["plan"]
    plan.set_precision("mixed")
    vm, rm = plan.assemble_linear(model.external_load_vector())
    um = solve(sysg.n_free, to_np(sysg.row_ptr), to_np(sysg.col_idx), to_np(vm), to_np(rm))
    assert rel_fro(um, uo) <= 1e-6


def test_prescribed_displacement_rhs(cuda, port):
    """Nonzero SPC values move -K_fc u_c into the rhs (src/fem/assembly.cpp:95-96)."""
    model = box_model(mg.C3D20, 2, 2, 1, jitter=0.05, seed=9, prescribe=0.01)
    sysg = assemble_linear_static(model)
    rp, ci, v, rhs = oracle_system(port, model)
    vgc, voc, _ = compare_patterns(to_np(sysg.row_ptr), to_np(sysg.col_idx), to_np(sysg.vals), rp, ci, v,
                                   sysg.n_free)
    assert rel_fro(vgc, voc) <= 1e-12
    assert rel_fro(to_np(sysg.rhs), rhs) <= 1e-12
    assert np.abs(rhs).max() > 0.0


def test_c3d20_lognormal_block(cuda, port):
    """Per-element lognormal E on a jittered C3D20 block (the 27-point benchmark case)."""
    cfg = mg.c3d20_block(4, seed=2)
    m = cfg["mesh"]
    model = Model(m, [Material(200000.0, 0.3)], None, cfg["spc"], None)
    f = cfg["f_ext"]
    plan = Plan(model)
    vg, rg = plan.assemble_linear(f)
    mats, em = per_element_materials(model)
    dof_eq, pre, nf = model.dof_map()
    rp, ci, v, rhs = port.assemble_linear(m, mats, em, dof_eq, pre, nf, f)
    rpg, cig = (to_np(t) for t in plan.pattern())
    vgc, voc, _ = compare_patterns(rpg, cig, to_np(vg), rp, ci, v, nf)
    assert rel_fro(vgc, voc) <= 1e-12
    ug = solve(nf, rpg, cig, to_np(vg), to_np(rg))
    uo = solve(nf, rp, ci, v, rhs)
    assert rel_fro(ug, uo) <= 1e-10


@pytest.mark.parametrize("etype,n", [(mg.C3D20, 6), (mg.C3D8, 10), (mg.C3D20R, 6), (mg.C3D15, 5), (mg.C3D6, 8)])
def test_mixed_precision_block_displacement(cuda, port, etype, n):
    """Mixed precision (FP32 Gram blocks, FP64 Jacobians / diagonal blocks / sums):
    displacement within 1e-6 relative L2 of the FP64 oracle on jittered blocks with
    lognormal E, z=0 clamped, unit shear load on the top face."""
    m = mg.box_mesh(etype, n, n, n, jitter=0.05, seed=etype)
    m.young = mg.lognormal_young(m.n_elems, seed=etype)
    m.poisson = np.full(m.n_elems, 0.3)
    top = mg.face_nodes(m, 2, 1.0)
    model = Model(m, [Material(200000.0, 0.3)], None, mg.clamp_face_spc(m, 2, 0.0),
                  (top, np.zeros(top.size, dtype=int), np.full(top.size, 1.0 / top.size)))
    rp, ci, v, rhs = oracle_system(port, model)
    uo = solve(len(rhs), rp, ci, v, rhs)
    plan = Plan(model, "mixed")
    vm, rm = plan.assemble_linear(model.external_load_vector())
    rpg, cig = (to_np(t) for t in plan.pattern())
    um = solve(plan.n_free, rpg, cig, to_np(vm), to_np(rm))
    assert rel_fro(um, uo) <= 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_repeat_assembly_bitwise_stable(cuda, precision):
    """Re-assembling into the same buffers gives the same bits: the row gather sums every
    CSR value in a fixed order with no atomics, so nothing may vary run to run."""
    model = box_model(mg.C3D8, 6, 4, 4, seed=5)
    plan = Plan(model, precision)
    v1, r1 = (to_np(t).copy() for t in plan.assemble_linear(model.external_load_vector()))
    v2, r2 = (to_np(t) for t in plan.assemble_linear(model.external_load_vector()))
    assert np.array_equal(v1, v2)
    assert np.array_equal(r1, r2)


def test_unknown_node_rejected(cuda):
    from calculixpp_b200 import CxgError
    model = box_model(mg.C3D8, 2, 1, 1)
    model.mesh.conn = model.mesh.conn.copy()
    model.mesh.conn[1, 3] = model.mesh.n_nodes + 5
    with pytest.raises(CxgError) as exc:
        Plan(model)
    assert exc.value.code == 6
    assert "unknown node" in str(exc.value)


def test_negative_jacobian_in_plan(cuda):
    from calculixpp_b200 import CxgError
    model = box_model(mg.C3D8, 2, 1, 1, jitter=0.0)
    model.mesh.conn = model.mesh.conn.copy()
    model.mesh.conn[1] = model.mesh.conn[1][[4, 5, 6, 7, 0, 1, 2, 3]]
    plan = Plan(model)
    with pytest.raises(CxgError) as exc:
        plan.assemble_linear()
    assert exc.value.code == 4
    assert "non-positive element Jacobian" in str(exc.value)


def _translation_residual(plan, n_nodes, vals):
    """max over rows of |K t| / max|K| for the three unit translations t (every DOF free)."""
    rp, ci = (to_np(t) for t in plan.pattern())
    K = sp.csr_matrix((to_np(vals), ci, rp), shape=(3 * n_nodes, 3 * n_nodes))
    worst = 0.0
    for d in range(3):
        t = np.zeros(3 * n_nodes)
        t[d::3] = 1.0
        worst = max(worst, np.abs(K @ t).max() / np.abs(K.data).max())
    return worst


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_mixed_rigid_translations_in_null_space(cuda, etype):
    """Mixed precision keeps the rigid translations in the null space of K to FP64
    rounding: the element pass forms each diagonal block in FP64 as minus the sum of the
    element row's FP32 off-diagonal blocks, so every assembled row sums to ~1e-16 of the
    largest entry, where FP32 diagonal blocks would leave ~1e-7. No constraint, so K is
    the full singular matrix."""
    quad = etype in (mg.C3D20, mg.C3D20R, mg.C3D15, mg.C3D10)
    dims = (3, 2, 2) if quad else (5, 3, 2)
    m = mg.box_mesh(etype, *dims, float(dims[0]), float(dims[1]), float(dims[2]), jitter=0.1, seed=etype)
    m.young = mg.lognormal_young(m.n_elems, seed=etype)
    m.poisson = np.full(m.n_elems, 0.3)
    none = (np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0))
    model = Model(m, [Material(200000.0, 0.3)], None, none, None)
    plan = Plan(model, "mixed")
    vals, _ = plan.assemble_linear(np.zeros(3 * m.n_nodes))
    assert _translation_residual(plan, m.n_nodes, vals) <= 1e-13


@pytest.mark.parametrize("etype", [mg.C3D8, mg.C3D8R, mg.C3D20])
def test_mixed_tangent_rigid_translations_in_null_space(cuda, etype):
    """The same for the consistent tangent of a J2 state with yielded points."""
    quad = etype == mg.C3D20
    n = 3 if quad else 5
    m = mg.box_mesh(etype, n, n, n, 1.0, 1.0, 1.0, jitter=0.05, seed=etype)
    m.young = np.full(m.n_elems, mg.J2_E)
    m.poisson = np.full(m.n_elems, mg.J2_NU)
    none = (np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0))
    model = Model(m, [Material(mg.J2_E, mg.J2_NU, mg.j2_table())], None, none, None)
    u = mg.graded_uniaxial_field(m.coords, 0.01)
    plan = Plan(model, "mixed")
    vals, _, _ = plan.assemble_tangent(u)
    ep = to_np(plan.state(committed=False))[:, 6]
    assert (ep > 0).mean() > 0.2  # yielded points take the plastic tangent
    assert _translation_residual(plan, m.n_nodes, vals) <= 1e-13
