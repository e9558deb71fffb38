"""Batched assembly of many independent models (cxg_batch_*): every model's slice of the
batch output equals the assembly of that model alone, bit for bit, in FP64 and mixed
precision, whatever launch shape the groups run with, directly or as a CUDA graph;
the autotuner's cache round-trips; J2 models assemble their tangent in the batch with
the same bits as alone."""
import ctypes as C
import json

import numpy as np
import pytest
import torch

from calculixpp_b200 import Batch, CxgError, Plan
from calculixpp_b200 import meshgen as mg
from calculixpp_b200.assembly import Material, Model
from tests.helpers import to_np

pytestmark = pytest.mark.gpu


def small_models(seed=0):
    rng = np.random.default_rng(seed)
    out = []
    types = [mg.C3D8, mg.C3D20R, mg.C3D6, mg.C3D8R, mg.C3D15, mg.C3D8, mg.C3D20, mg.C3D15, mg.C3D6, mg.C3D20R]
    for k, t in enumerate(types):
        ne = int(rng.integers(8, 300))
        E, nu = float(rng.uniform(7e4, 2.1e5)), float(rng.uniform(0.25, 0.35))
        m, spc, top = mg.batch_box(t, ne, 0.1, seed * 1000 + k, E, nu)
        if k % 3 == 0:
            m.young = m.young * rng.uniform(0.5, 1.5, m.n_elems)
        loads = (top, np.zeros(top.size, dtype=np.int64), np.full(top.size, 1.0 / top.size))
        out.append(Model(m, [Material(E, nu)], None, spc, loads))
    return out


@pytest.fixture(scope="module")
def models():
    return small_models()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_single_model_plans(cuda, models, precision):
    b = Batch(models, precision)
    f = torch.as_tensor(b.load_vector(), device=b.device)
    vals, rhs = b.assemble(f)
    assert b.n_groups == len({m.mesh.etype for m in models})
    for k, model in enumerate(models):
        plan = Plan(model, precision)
        v1, r1 = plan.assemble_linear(model.external_load_vector())
        vk, rk = b.slices(k, vals, rhs)
        rp, ci = b.pattern(k)
        rp1, ci1 = (to_np(t) for t in plan.pattern())
        assert np.array_equal(rp, rp1) and np.array_equal(ci, ci1)
        assert torch.equal(vk, v1), k
        assert torch.equal(rk, r1), k
        plan.close()
    b.close()


def test_graph_launch_and_tile_shapes(cuda, models):
    b = Batch(models, "mixed")
    f = torch.as_tensor(b.load_vector(), device=b.device)
    ref_v, ref_r = b.assemble(f)
    ref_v, ref_r = ref_v.clone(), ref_r.clone()
    vals, rhs = b.buffers()
    for _ in range(3):
        vals.fill_(np.nan)
        b.graph_launch(f, vals, rhs, check=True)
    assert torch.equal(vals, ref_v) and torch.equal(rhs, ref_r)
    # every tile shape and launch shape gives the same bits (graph re-captured on change)
    for tile in (1, 2):
        for g in range(b.n_groups):
            b.set_group_config(g, tile=tile, p1_blocks_per_sm=1, p2_warps=4)
        vals.zero_()
        b.graph_launch(f, vals, rhs, check=True)
        assert torch.equal(vals, ref_v), tile
    b.set_precision("fp64")
    with pytest.raises(CxgError):
        b.set_group_config(0, tile=2)
    b.close()


def test_tuner_cache_round_trip(cuda, models, tmp_path):
    b = Batch(models, "mixed")
    f = torch.as_tensor(b.load_vector(), device=b.device)
    ref_v, ref_r = (t.clone() for t in b.assemble(f))
    vals, rhs = b.buffers()
    cache = tmp_path / "tune.json"
    cfg = b.tune(f, vals, rhs, cache)
    assert torch.equal(vals, ref_v) and torch.equal(rhs, ref_r)
    data = json.loads(cache.read_text())
    assert len(data) == b.n_groups
    for key, entry in data.items():
        assert key.startswith("sm") and "/mixed/" in key
        assert entry["tile"] in (0, 1, 2) and entry["p2_warps"] in (2, 4, 8) and entry["p1_ms"] > 0
    # a second batch reads the cache instead of measuring, and picks the same shapes
    b2 = Batch(models, "mixed")
    before = cache.read_text()
    assert b2.tune(f, vals, rhs, cache) == cfg
    assert cache.read_text() == before
    b.close()
    b2.close()


def test_host_buffers_and_rejections(cuda, models):
    b = Batch(models[:3], "fp64")
    f = b.load_vector()
    hv = torch.empty(b.nnz, dtype=torch.float64)
    hr = torch.empty(b.n_free, dtype=torch.float64)
    b.assemble(torch.as_tensor(f), hv, hr)
    dv, dr = b.assemble(torch.as_tensor(f, device=b.device))
    assert torch.equal(hv, dv.cpu()) and torch.equal(hr, dr.cpu())
    b.close()
    b2 = Batch(models[:2], "fp64")
    hu = np.zeros(3 * b2.n_nodes)  # host u: the batched tangent takes device buffers only
    vals, rhs = b2.buffers()
    rc = b2.lib.cxg_batch_assemble_tangent(b2.h, C.c_void_p(hu.ctypes.data), C.c_void_p(vals.data_ptr()), None,
                                           C.c_void_p(rhs.data_ptr()), None, None)
    assert rc == 1 and b"device buffers" in b2.lib.cxg_last_error()
    b2.close()


J2 = ([0.0, 1.0], [250.0, 1250.0])  # sigma_y 250, linear hardening H = 1000


def plastic_models(seed=4):
    rng = np.random.default_rng(seed)
    out = []
    for k, t in enumerate([mg.C3D8, mg.C3D20R, mg.C3D6, mg.C3D8R, mg.C3D15, mg.C3D8]):
        ne = int(rng.integers(20, 200))
        E, nu = float(rng.uniform(7e4, 2.1e5)), float(rng.uniform(0.25, 0.35))
        m, spc, top = mg.batch_box(t, ne, 0.1, seed * 1000 + k, E, nu)
        mats = [Material(E, nu, J2)] if k % 2 == 0 else [Material(E, nu), Material(E, nu, J2, 2, 3000.0)]
        em = None if k % 2 == 0 else (np.arange(m.n_elems) % 2).astype(np.int32)
        out.append(Model(m, mats, em, spc, None))
    return out


def _u(model, scale):
    x = model.mesh.coords
    h = x[:, 2].max()
    u = np.zeros_like(x)
    u[:, 0] = scale * x[:, 2] * (1.0 + 0.3 * x[:, 0] / max(x[:, 0].max(), 1.0))
    u[:, 2] = 0.4 * scale * x[:, 2] ** 2 / h
    return u.reshape(-1)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_plastic_models_equal_single_plans(cuda, precision):
    """J2 models of several types (isotropic and combined hardening, per-element
    materials) in one batch: every model's tangent, internal force, rhs and history equal
    those of a plan of that model alone, bit for bit, over two increments with commits."""
    models = plastic_models()
    b = Batch(models, precision)
    plans = [Plan(m, precision) for m in models]
    vals, rhs = b.buffers()
    for step, scale in enumerate((0.004, 0.009)):
        u = torch.as_tensor(b.displacement_vector([_u(m, scale) for m in models]), device=b.device)
        vals, f_int, rhs = b.assemble_tangent(u, vals=vals, rhs=rhs)
        for k, (model, plan) in enumerate(zip(models, plans)):
            v1, f1, r1 = plan.assemble_tangent(_u(model, scale))
            vk, rk = b.slices(k, vals, rhs)
            assert torch.equal(vk, v1), (step, k)
            assert torch.equal(rk, r1), (step, k)
            assert torch.equal(b.f_int_slice(k, f_int), f1), (step, k)
            assert torch.equal(b.state(k, committed=False), plan.state(committed=False)), (step, k)
        b.commit()
        for plan in plans:
            plan.commit()
    assert any(float(b.state(k)[:, 6].max()) > 0.0 for k in range(len(models)))  # yielded
    for plan in plans:
        plan.close()
    b.close()
