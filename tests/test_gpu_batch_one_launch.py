"""One-launch batches (cxg_batch_set_launch(CXG_BATCH_ONE_LAUNCH)): the whole batch is one
element pass and one row gather, every element-type group a slot of the same two
kernels. Every output equals the per-group launches' bit for bit, directly, as a CUDA
graph, at every tile it takes and after tuning, for linear and J2 (material-point)
assembly over committed increments."""
import ctypes as C
import json

import numpy as np
import pytest
import torch

from calculixpp_b200 import Batch, CxgError
from tests.test_gpu_batch import _u, plastic_models, small_models

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def models():
    return small_models(seed=3)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_one_launch_equals_per_group(cuda, models, precision):
    b = Batch(models, precision)
    assert b.launch_mode() == "per_group"
    f = torch.as_tensor(b.load_vector(), device=b.device)
    ref_v, ref_r = (t.clone() for t in b.assemble(f))
    b.set_launch("one_launch")
    assert b.launch_mode() == "one_launch"
    vals, rhs = b.buffers()
    vals.fill_(np.nan)
    rhs.fill_(np.nan)
    b.assemble(f, vals, rhs)
    assert torch.equal(vals, ref_v) and torch.equal(rhs, ref_r)
    for _ in range(2):
        vals.fill_(np.nan)
        b.graph_launch(f, vals, rhs, check=True)
        assert torch.equal(vals, ref_v) and torch.equal(rhs, ref_r)
    # the tiles the one-launch element pass takes, pinned per group (graph re-captured)
    tiles = (1, 0) if precision == "mixed" else (1,)
    for tile in tiles:
        for g in range(b.n_groups):
            b.set_group_config(g, tile=tile, p2_warps=4)
            assert b.group_config(g)["tile"] == {0: "2x4", 1: "2x2"}[tile]
        vals.zero_()
        b.graph_launch(f, vals, rhs, check=True)
        assert torch.equal(vals, ref_v), tile
    if precision == "fp64":
        with pytest.raises(CxgError):
            b.set_group_config(0, tile=0)  # 2x4 FP64 accumulators do not fit the shared kernel
    b.close()


def test_one_launch_tuner_and_cache(cuda, models, tmp_path):
    b = Batch(models, "mixed")
    f = torch.as_tensor(b.load_vector(), device=b.device)
    ref_v, ref_r = (t.clone() for t in b.assemble(f))
    b.set_launch("one_launch")
    vals, rhs = b.buffers()
    cache = tmp_path / "tune.json"
    cfg = b.tune(f, vals, rhs, cache)
    assert torch.equal(vals, ref_v) and torch.equal(rhs, ref_r)
    data = json.loads(cache.read_text())
    assert len(data) == b.n_groups and all(k.endswith("/one-launch") for k in data)
    for entry in data.values():
        assert entry["tile"] in (0, 1) and entry["p2_warps"] in (2, 4, 8)
        assert entry["p1_ms"] > 0 and entry["p2_ms"] > 0
    b2 = Batch(models, "mixed")
    b2.set_launch("one_launch")
    before = cache.read_text()
    assert b2.tune(f, vals, rhs, cache) == cfg
    assert cache.read_text() == before
    vals.zero_()
    b2.graph_launch(f, vals, rhs, check=True)
    assert torch.equal(vals, ref_v) and torch.equal(rhs, ref_r)
    b.close()
    b2.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_one_launch_plastic_batch_equals_per_group(cuda, precision):
    """J2 models of several types: tangent, internal force, rhs and history of the one
    launch equal the per-group launches' over two increments with commits."""
    models = plastic_models()
    a = Batch(models, precision)
    b = Batch(models, precision)
    b.set_launch("one_launch")
    va, ra = a.buffers()
    vb, rb = b.buffers()
    for step, scale in enumerate((0.004, 0.009)):
        u = torch.as_tensor(a.displacement_vector([_u(m, scale) for m in models]), device=a.device)
        va, fa, ra = a.assemble_tangent(u, vals=va, rhs=ra)
        vb.fill_(np.nan)
        vb, fb, rb = b.assemble_tangent(u, vals=vb, rhs=rb)
        assert torch.equal(va, vb) and torch.equal(ra, rb) and torch.equal(fa, fb), step
        for k in range(len(models)):
            assert torch.equal(a.state(k, committed=False), b.state(k, committed=False)), (step, k)
        a.commit()
        b.commit()
    assert any(float(b.state(k)[:, 6].max()) > 0.0 for k in range(len(models)))  # yielded
    a.close()
    b.close()


def test_launch_mode_rejections(cuda, models):
    b = Batch(models[:2], "fp64")
    assert b.lib.cxg_batch_set_launch(b.h, 7) == 1
    assert b"launch mode" in b.lib.cxg_last_error()
    mode = C.c_int32(-1)
    assert b.lib.cxg_batch_get_launch(b.h, C.byref(mode)) == 0 and mode.value == 0
    b.close()
