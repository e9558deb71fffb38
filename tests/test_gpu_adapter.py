"""The C++ seam: calculixpp_b200/adapter/cxg_cxpp.cpp compiled against the reference's
headers and linked with the reference itself (oracle/_ref/libcxg_cxpp_test.so). The
reference's own linear-static pipeline (solver choice, solve_reduced through the compute
backend, expansion through the constraint transform, field recovery) runs on the
LinearSystem the adapter assembles on the GPU, and is compared with the same pipeline
all on the CPU (numerics::solve_linear_static), on the same Model object:

* displacements within 1e-10 relative L2, nodal stress within 1e-9 (FP64 assembly);
  displacements within 1e-6 with the mixed-precision assembly;
* the LinearSystem itself: the same triplets (as canonical CSR) within 1e-12, the same rhs;
* the material-point path (J2, per-element sections): tangent and f_int within 1e-12
  over three increments with commits, against assemble_material_tangent;
* *EQUATION constraints (slave elimination through the reference's constraint
  transform, including a slave whose master is a nonzero SPC): the reduced system within
  1e-12, displacements within 1e-10, the J2 tangent within 1e-12;
* models the GPU path does not cover (several element types) raise the adapter's
  message instead of returning a wrong system;
* CudaBackend (ComputeBackend::solve_sparse on the device): duplicate COO entries summed,
  the direct solve within 1e-10 and CG within 1e-8 of a host direct solve, and the whole
  linear-static pipeline with the assembly and the solve on the GPU.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from calculixpp_b200 import meshgen as mg
from oracle.oracle import Material, OracleError, RefCuda, coo_to_csr, make_material
from tests.helpers import rel_fro

pytestmark = pytest.mark.gpu

ISO = ([0.0, 0.02], [800.0, 960.0])


@pytest.fixture(scope="module")
def adapter(ref):
    if not RefCuda.available():
        pytest.skip("adapter library oracle/_ref/libcxg_cxpp_test.so not built")
    return RefCuda()


def _cantilever(etype, dims, seed):
    nx, ny, nz = dims
    m = mg.box_mesh(etype, nx, ny, nz, float(nx), float(ny), float(nz), jitter=0.08, seed=seed)
    sn, sc, sv = mg.clamp_face_spc(m, 0, 0.0)
    tip = mg.face_nodes(m, 0, float(nx))
    cl = (tip, np.full(tip.size, 2), np.full(tip.size, -100.0 / tip.size))
    # two sections: the far half of the elements gets a second material
    centre_x = m.coords[m.conn].mean(axis=1)[:, 0]
    elem_mat = (centre_x > nx / 2).astype(np.int32)
    return m, (sn, sc, sv), cl, elem_mat


def _csr_on(ref_rp, ref_ci, nf, rows, cols, vals):
    """The adapter's triplets as canonical CSR restricted to the reference's pattern (the
    entries the reference leaves out must be below rounding)."""
    rp, ci, v = coo_to_csr(nf, rows, cols, vals)
    if np.array_equal(rp, ref_rp) and np.array_equal(ci, ref_ci):
        return v
    kg = np.repeat(np.arange(nf), np.diff(rp)).astype(np.int64) * nf + ci
    ko = np.repeat(np.arange(nf), np.diff(ref_rp)).astype(np.int64) * nf + ref_ci
    keep = np.isin(kg, ko)
    assert keep.sum() == ko.size
    assert np.abs(v[~keep]).max() <= 1e-12 * np.abs(v).max()
    return v[keep]


@pytest.mark.parametrize("etype", [mg.C3D8, mg.C3D20, mg.C3D6, mg.C3D10])
def test_solve_linear_static_on_gpu_assembly(cuda, ref, adapter, etype):
    quad = etype in (mg.C3D20, mg.C3D10)
    m, spc, cl, em = _cantilever(etype, (4, 2, 2) if quad else (8, 3, 3), seed=etype)
    mats = [make_material(210000.0, 0.3), make_material(70000.0, 0.33)]
    rm = ref.model(m, mats, em, spc, cl)
    u_cpu, s_cpu = adapter.solve_linear_static(rm, gpu=0)
    u_gpu, s_gpu = adapter.solve_linear_static(rm, gpu=1)
    assert rel_fro(u_gpu, u_cpu) <= 1e-10
    assert rel_fro(s_gpu, s_cpu) <= 1e-9
    u_mx, _ = adapter.solve_linear_static(rm, gpu=1, precision=1)
    assert rel_fro(u_mx, u_cpu) <= 1e-6


@pytest.mark.parametrize("etype", [mg.C3D8, mg.C3D20])
def test_thermal_strain_model(cuda, ref, adapter, etype):
    """A model with *EXPANSION (a constant alpha on one section, an alpha(T) table on the
    other) and temperatures applied on part of the nodes: the adapter passes the reference
    model's own thermal inputs to the plan, so the linear system's rhs carries the
    thermal-strain load (assemble_linear_static, src/fem/assembly.cpp:251-253) and the
    solve agrees with the reference pipeline on the CPU."""
    quad = etype == mg.C3D20
    m, spc, cl, em = _cantilever(etype, (4, 2, 2) if quad else (8, 3, 3), seed=30 + etype)
    mats = [make_material(210000.0, 0.3), make_material(70000.0, 0.33)]
    rm = ref.model(m, mats, em, spc, cl)
    rm.set_expansion([([1.2e-5], [0.0]), ([1.0e-5, 2.0e-5], [0.0, 300.0])], [20.0, 0.0])
    rng = np.random.default_rng(etype)
    nodes = np.flatnonzero(rng.uniform(size=m.n_nodes) < 0.8)
    rm.set_temperature(nodes, rng.uniform(50.0, 250.0, nodes.size))
    want = rm.assemble_linear_static()
    h = adapter.assembler(rm)
    try:
        _, _, _, rhs = adapter.assemble_linear(h)
    finally:
        adapter.free(h)
    assert rel_fro(rhs, want["rhs"]) <= 1e-12
    u_cpu, s_cpu = adapter.solve_linear_static(rm, gpu=0)
    u_gpu, s_gpu = adapter.solve_linear_static(rm, gpu=1)
    assert rel_fro(u_gpu, u_cpu) <= 1e-10
    assert rel_fro(s_gpu, s_cpu) <= 1e-9


@pytest.mark.parametrize("etype", [mg.C3D8, mg.C3D8R, mg.C3D20R, mg.C3D15])
def test_linear_system_matches_reference(cuda, ref, adapter, etype):
    quad = etype in (mg.C3D20R, mg.C3D15)
    m, spc, cl, em = _cantilever(etype, (3, 2, 2) if quad else (6, 3, 2), seed=10 + etype)
    mats = [make_material(210000.0, 0.3), make_material(120000.0, 0.28)]
    rm = ref.model(m, mats, em, spc, cl)
    want = rm.assemble_linear_static()
    nf = want["n_free"]
    rp, ci, v = coo_to_csr(nf, want["rows"], want["cols"], want["vals"])
    h = adapter.assembler(rm)
    try:
        rows, cols, vals, rhs = adapter.assemble_linear(h)
    finally:
        adapter.free(h)
    assert np.all(np.diff(rows.astype(np.int64) * nf + cols) > 0)  # (row, column) order, duplicates summed
    assert rel_fro(_csr_on(rp, ci, nf, rows, cols, vals), v) <= 1e-12
    assert rel_fro(rhs, want["rhs"]) <= 1e-12


def test_material_tangent_matches_reference(cuda, ref, adapter):
    m, spc, _, em = _cantilever(mg.C3D8, (6, 2, 2), seed=3)
    mats = [make_material(210000.0, 0.3, ISO, 0), make_material(200000.0, 0.29, ([0.0, 0.01], [600.0, 700.0]), 0)]
    rm = ref.model(m, mats, em, spc, None)
    h = adapter.assembler(rm)
    try:
        x = m.coords
        for k in range(1, 4):
            u = np.zeros_like(x)
            u[:, 0] = 0.004 * k * x[:, 0] * (0.3 + x[:, 2] / x[:, 2].max())
            u[:, 2] = -0.002 * k * x[:, 0] ** 2 / x[:, 0].max()
            u = u.reshape(-1)
            want = rm.assemble_material_tangent(u)
            rm.commit()
            rows, cols, vals, rhs, f_int = adapter.assemble_tangent(h, u, commit=True)
            nf = want["n_free"]
            rp, ci, v = coo_to_csr(nf, want["rows"], want["cols"], want["vals"])
            assert rel_fro(_csr_on(rp, ci, nf, rows, cols, vals), v) <= 1e-12, k
            assert rel_fro(f_int, want["f_int"]) <= 1e-12, k
            assert rel_fro(rhs, want["rhs"]) <= 1e-12, k
        assert np.any(rm.state()[6::13] > 0.0)  # yielded
    finally:
        adapter.free(h)


def test_several_element_types_rejected(cuda, ref, adapter):
    a = mg.box_mesh(mg.C3D8, 2, 1, 1, 2.0, 1.0, 1.0)
    b = mg.box_mesh(mg.C3D6, 1, 1, 1, 1.0, 1.0, 1.0)
    coords = np.ascontiguousarray(np.concatenate([a.coords, b.coords + np.array([5.0, 0.0, 0.0])]))
    types = np.concatenate([np.full(a.n_elems, mg.C3D8), np.full(b.n_elems, mg.C3D6)]).astype(np.int32)
    conn = np.concatenate([a.conn.ravel(), (b.conn + a.n_nodes).ravel()]).astype(np.int32)
    conn_ptr = np.concatenate([[0], np.cumsum([8] * a.n_elems + [6] * b.n_elems)]).astype(np.int64)
    E = a.n_elems + b.n_elems
    em = np.zeros(E, np.int32)
    mats = (Material * 1)(make_material(210000.0, 0.3))
    zi, zd = np.zeros(1, np.int32), np.zeros(1)
    h = ref._fn("model_create")(coords.shape[0], coords.ctypes.data, E, types.ctypes.data, conn_ptr.ctypes.data,
                                conn.ctypes.data, em.ctypes.data, 1, mats, 0, zi.ctypes.data, zi.ctypes.data,
                                zd.ctypes.data, 0, zi.ctypes.data, zi.ctypes.data, zd.ctypes.data)
    assert h

    class _Handle:
        pass

    rm = _Handle()
    rm.h = h
    try:
        with pytest.raises(OracleError, match="several element types"):
            adapter.assembler(rm)
    finally:
        ref._fn("model_free")(C.c_void_p(h))


def _with_equations(ref, etype, plastic=False):
    """Cantilever with *EQUATION ties: the tip face's z motion follows its first node,
    and the y motion of a node near the centre is half that of a node whose y is
    prescribed to a nonzero value (the expansion's constant goes to the rhs)."""
    m, (sn, sc, sv), cl, em = _cantilever(etype, (6, 2, 2) if etype == mg.C3D8 else (3, 2, 2), seed=21)
    tip = mg.face_nodes(m, 0, float(6 if etype == mg.C3D8 else 3))
    mid = int(np.argmin(np.abs(m.coords - m.coords.mean(axis=0)).sum(axis=1)))
    pres_node = int(tip[-1])
    sn = np.concatenate([sn, [pres_node]]).astype(np.int32)
    sc = np.concatenate([sc, [1]]).astype(np.int32)
    sv = np.concatenate([sv, [0.02]])
    mats = ([make_material(210000.0, 0.3, ISO, 0), make_material(150000.0, 0.3, ISO, 0)] if plastic
            else [make_material(210000.0, 0.3), make_material(70000.0, 0.33)])
    rm = ref.model(m, mats, em, (sn, sc, sv), cl)
    for node in tip[1:-1]:
        rm.add_equation([int(node), int(tip[0])], [2, 2], [1.0, -1.0])
    rm.add_equation([mid, pres_node], [1, 1], [2.0, -1.0])  # u_y(mid) = u_y(prescribed node) / 2
    return m, rm


@pytest.mark.parametrize("etype", [mg.C3D8, mg.C3D20])
def test_equations_linear_system_and_solve(cuda, ref, adapter, etype):
    m, rm = _with_equations(ref, etype)
    want = rm.assemble_linear_static()
    nf = want["n_free"]
    assert nf < 3 * m.n_nodes - 3 * mg.face_nodes(m, 0, 0.0).size - 1  # slaves eliminated
    rp, ci, v = coo_to_csr(nf, want["rows"], want["cols"], want["vals"])
    h = adapter.assembler(rm)
    try:
        rows, cols, vals, rhs = adapter.assemble_linear(h)
    finally:
        adapter.free(h)
    assert rel_fro(_csr_on(rp, ci, nf, rows, cols, vals), v) <= 1e-12
    assert rel_fro(rhs, want["rhs"]) <= 1e-12
    u_cpu, _ = adapter.solve_linear_static(rm, gpu=0)
    u_gpu, _ = adapter.solve_linear_static(rm, gpu=1)
    assert rel_fro(u_gpu, u_cpu) <= 1e-10


def test_equations_material_tangent(cuda, ref, adapter):
    m, rm = _with_equations(ref, mg.C3D8, plastic=True)
    h = adapter.assembler(rm)
    try:
        x = m.coords
        for k in (1, 2):
            u = np.zeros_like(x)
            u[:, 0] = 0.004 * k * x[:, 0] * (0.3 + x[:, 2] / x[:, 2].max())
            u = u.reshape(-1)
            want = rm.assemble_material_tangent(u)
            rm.commit()
            rows, cols, vals, rhs, f_int = adapter.assemble_tangent(h, u, commit=True)
            nf = want["n_free"]
            rp, ci, v = coo_to_csr(nf, want["rows"], want["cols"], want["vals"])
            assert rel_fro(_csr_on(rp, ci, nf, rows, cols, vals), v) <= 1e-12, k
            assert rel_fro(f_int, want["f_int"]) <= 1e-12, k
            assert rel_fro(rhs, want["rhs"]) <= 1e-12, k
    finally:
        adapter.free(h)


def test_cuda_backend_solve_sparse(cuda, ref, adapter):
    """CudaBackend::solve_sparse on a reference LinearSystem's COO triplets, with part of
    the entries split into duplicate triplets (summed like the CPU backend's from_coo):
    the direct solve within 1e-10 of a host direct solve, CG within 1e-8."""
    import scipy.sparse.linalg as spla
    m, spc, cl, em = _cantilever(mg.C3D8, (8, 3, 3), seed=5)
    rm = ref.model(m, [make_material(210000.0, 0.3), make_material(70000.0, 0.33)], em, spc, cl)
    sys_ = rm.assemble_linear_static()
    nf = sys_["n_free"]
    rows, cols, vals = sys_["rows"], sys_["cols"], sys_["vals"].copy()
    split = np.arange(0, vals.size, 3)
    half = 0.5 * vals[split]
    vals[split] -= half
    rows2 = np.concatenate([rows, rows[split]])
    cols2 = np.concatenate([cols, cols[split]])
    vals2 = np.concatenate([vals, half])
    A = sp.coo_matrix((sys_["vals"], (rows, cols)), shape=(nf, nf)).tocsc()
    want = spla.spsolve(A, sys_["rhs"])
    x_direct = adapter.backend_solve(nf, rows2, cols2, vals2, sys_["rhs"], solver=0)
    assert rel_fro(x_direct, want) <= 1e-10
    x_cg = adapter.backend_solve(nf, rows2, cols2, vals2, sys_["rhs"], solver=1)
    assert rel_fro(x_cg, want) <= 1e-8


@pytest.mark.parametrize("solver", [0, 1])
def test_linear_static_all_on_gpu(cuda, ref, adapter, solver):
    """solve_linear_static with the assembly and the solve on the GPU against the same
    pipeline all on the CPU (direct solve there)."""
    m, spc, cl, em = _cantilever(mg.C3D20, (4, 2, 2), seed=9)
    rm = ref.model(m, [make_material(210000.0, 0.3), make_material(70000.0, 0.33)], em, spc, cl)
    u_cpu, _ = adapter.solve_linear_static(rm, gpu=0)
    u_gpu, _ = adapter.solve_linear_static(rm, gpu=2, solver=solver)
    assert rel_fro(u_gpu, u_cpu) <= (1e-10 if solver == 0 else 1e-8)
