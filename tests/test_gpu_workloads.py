"""Parity of the CUDA path against the oracle on the benchmark's own workload generators,
at sizes the oracle finishes in seconds:

* the J2 Newton workload (C3D8 block, graded uniaxial ramp, `c3d8_j2_block` +
  `j2_increment`) through all 10 increments with a commit after each: FP64 tangent and
  f_int within 1e-12 relative, J2 history within 1e-10 per Gauss point; the mixed path's
  K and f_int against the same oracle within 1e-6, its history (FP64 return) equal to
  the FP64 path's bit for bit, and with the FP32 return K and f_int within 1e-6 and the
  history within 1e-5 of its magnitude;
* the C3D20 block (`c3d20_block`, lognormal E): CSR pattern bit-exact, FP64 values within
  1e-12, displacements within 1e-10 after the same direct solve; mixed displacements
  within 1e-6 of the oracle's;
* 16 models of the batched workload (`batched_workload`), every model's slice of the
  batch against the oracle's assembly of that model alone (1e-12 in FP64; 1e-6
  displacement in mixed precision);
* the adjoint workload (`adjoint_cantilever`, E = E0 rho^3) at 8x8x4: dc/drho through the
  autograd function against central differences of the compliance (step 1e-6 relative).
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

from calculixpp_b200 import Batch, Plan
from calculixpp_b200 import meshgen as mg
from calculixpp_b200.adjoint import compliance
from calculixpp_b200.assembly import Material, Model
from oracle.oracle import make_material
from tests.helpers import per_element_materials, rel_fro, to_np

pytestmark = pytest.mark.gpu


def _on_oracle_pattern(plan, vals, rp, ci):
    """GPU values restricted to the oracle's pattern; the pattern must contain it and
    the entries the oracle leaves out (every contribution exactly 0.0 there) must be
    below rounding (FP64 rounding, or FP32 rounding of the blocks in mixed precision)."""
    rpg, cig = (to_np(t) for t in plan.pattern())
    v = to_np(vals)
    if np.array_equal(rpg, rp) and np.array_equal(cig, ci):
        return v
    nf = rp.size - 1
    kg = np.repeat(np.arange(nf), np.diff(rpg)).astype(np.int64) * nf + cig
    ko = np.repeat(np.arange(nf), np.diff(rp)).astype(np.int64) * nf + ci
    keep = np.isin(kg, ko)
    assert keep.sum() == ko.size
    extra = 1e-12 if plan.precision == "fp64" else 1e-6
    assert np.abs(v[~keep]).max(initial=0.0) <= extra * np.abs(v).max()
    return v[keep]


def _solve(n, rp, ci, v, rhs):
    A = sp.csr_matrix((v, ci, rp), shape=(n, n))
    return spla.spsolve(A.tocsc(), rhs)


def test_j2_workload_ramp(cuda, port):
    n = 12
    cfg = mg.c3d8_j2_block(n)
    m = cfg["mesh"]
    mats_dev = [Material(mg.J2_E, mg.J2_NU, cfg["table"])]
    u1, spc1 = mg.j2_increment(cfg, 1)
    model = Model(m, mats_dev, None, spc1, None)
    plan64 = Plan(model, "fp64")
    planmx = Plan(model, "mixed")
    planf32 = Plan(model, "mixed")
    planf32.set_j2_fp32_return(True)
    mats, em = per_element_materials(model)
    dof_eq, pre, nf = model.dof_map()
    committed = np.zeros(plan64.n_gauss * 13)
    for k in range(1, 11):
        u, _ = mg.j2_increment(cfg, k)
        rp, ci, vo, rhs_o, fo, so = port.assemble_tangent(m, mats, em, dof_eq, pre, nf, u, committed)
        v64, f64, _ = plan64.assemble_tangent(u)
        assert rel_fro(_on_oracle_pattern(plan64, v64, rp, ci), vo) <= 1e-12, k
        assert rel_fro(to_np(f64), fo) <= 1e-12, k
        s64 = to_np(plan64.state(committed=False)).reshape(-1)
        assert np.all(np.abs(s64 - so) <= 1e-10 * np.maximum(1.0, np.abs(so))), k
        vmx, fmx, _ = planmx.assemble_tangent(u)
        assert rel_fro(_on_oracle_pattern(planmx, vmx, rp, ci), vo) <= 1e-6, k
        assert rel_fro(to_np(fmx), fo) <= 1e-6, k
        assert np.array_equal(to_np(planmx.state(committed=False)).reshape(-1), s64), k
        vf, ff, _ = planf32.assemble_tangent(u)
        assert rel_fro(_on_oracle_pattern(planf32, vf, rp, ci), vo) <= 1e-6, k
        assert rel_fro(to_np(ff), fo) <= 1e-6, k
        sf = to_np(planf32.state(committed=False)).reshape(-1)
        # FP32 Newton increments: ~1e-6 relative error of the increment
        assert np.abs(sf - so).max() <= 1e-5 * max(np.abs(so).max(), 1e-12), k
        plan64.commit()
        planmx.commit()
        planf32.commit()
        committed = so
    yielded = np.mean(committed.reshape(-1, 13)[:, 6] > 0)
    assert 0.2 < yielded < 0.6, yielded  # the ramp yields part of the block (~40 % at full size)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_c3d20_workload_block(cuda, port, precision):
    cfg = mg.c3d20_block(6, seed=3)
    m = cfg["mesh"]
    model = Model(m, [Material(200000.0, 0.3)], None, cfg["spc"], None)
    mats, em = per_element_materials(model)
    dof_eq, pre, nf = model.dof_map()
    rp, ci, vo, rhs_o = port.assemble_linear(m, mats, em, dof_eq, pre, nf, cfg["f_ext"])
    plan = Plan(model, precision)
    vg, rg = plan.assemble_linear(cfg["f_ext"])
    rpg, cig = (to_np(t) for t in plan.pattern())
    assert np.array_equal(rpg, rp) and np.array_equal(cig, ci)
    uo = _solve(nf, rp, ci, vo, rhs_o)
    ug = _solve(nf, rpg, cig, to_np(vg), to_np(rg))
    if precision == "fp64":
        assert rel_fro(to_np(vg), vo) <= 1e-12
        assert rel_fro(to_np(rg), rhs_o) <= 1e-12
        assert rel_fro(ug, uo) <= 1e-10
    else:
        assert rel_fro(ug, uo) <= 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_workload_slices(cuda, port, precision):
    work = mg.batched_workload(16, min_elems=100, max_elems=2000, seed=7)
    models = [Model(mm, [Material(E, nu)], None, spc,
                    (top, np.zeros(top.size, np.int64), np.full(top.size, 1.0 / top.size)))
              for mm, spc, top, E, nu in work]
    b = Batch(models, precision)
    f = torch.as_tensor(b.load_vector(), device=b.device)
    vals, rhs = b.graph_launch(f, *b.buffers(), check=True)
    torch.cuda.synchronize()
    for k, model in enumerate(models):
        mm = model.mesh
        dof_eq, pre, nf = model.dof_map()
        rp, ci, vo, rhs_o = port.assemble_linear(mm, [make_material(model.materials[0].E, model.materials[0].nu)],
                                                 None, dof_eq, pre, nf, model.external_load_vector())
        vk, rk = b.slices(k, vals, rhs)
        rpb, cib = b.pattern(k)
        nfk = rp.size - 1
        kb = np.repeat(np.arange(nfk), np.diff(rpb)).astype(np.int64) * nfk + cib
        ko = np.repeat(np.arange(nfk), np.diff(rp)).astype(np.int64) * nfk + ci
        keep = np.isin(kb, ko)
        assert keep.sum() == ko.size, k
        v = to_np(vk)
        # entries the reference leaves out (all contributions exactly 0.0 there) are zero
        # to rounding: FP64 rounding, or FP32 rounding of the blocks in mixed precision
        extra = 1e-12 if precision == "fp64" else 1e-6
        assert np.abs(v[~keep]).max(initial=0.0) <= extra * np.abs(v).max(), k
        if precision == "fp64":
            assert rel_fro(v[keep], vo) <= 1e-12, k
            assert rel_fro(to_np(rk), rhs_o) <= 1e-12, k
        else:
            uo = _solve(nfk, rp, ci, vo, rhs_o)
            ub = _solve(nfk, rpb, cib, v, to_np(rk))
            assert rel_fro(ub, uo) <= 1e-6, (k, mg.TYPE_NAMES[mm.etype])
    b.close()


def test_adjoint_workload_central_differences(cuda):
    cfg = mg.adjoint_cantilever(8, 8, 4, seed=2)
    m = cfg["mesh"]
    model = Model(m, [Material(210000.0, 0.3)], None, cfg["spc"], cfg["cloads"])
    plan = Plan(model)
    f = model.external_load_vector()
    dev = plan.device
    rho = torch.as_tensor(cfg["rho"], device=dev).requires_grad_(True)
    X = torch.as_tensor(m.coords, device=dev)
    c = compliance(210000.0 * rho ** 3, X, plan, f)
    (g,) = torch.autograd.grad(c, (rho,))

    def c_at(r):
        with torch.no_grad():
            return float(compliance(210000.0 * r ** 3, X, plan, f))

    rng = np.random.default_rng(3)
    cg_noise = 4 * 1e-12 * abs(float(c))
    for k in rng.choice(m.n_elems, 64, replace=False):
        h = 1e-6 * float(rho[k])
        rp, rm = rho.detach().clone(), rho.detach().clone()
        rp[k] += h
        rm[k] -= h
        fd = (c_at(rp) - c_at(rm)) / (2 * h)
        gk = float(g[k])
        assert abs(fd - gk) <= 1e-5 * abs(gk) + cg_noise / h, (k, fd, gk)
