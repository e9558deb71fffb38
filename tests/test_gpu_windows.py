"""Windowed assembly (cxg_plan_set_ring_bytes): the element pass and the row gather run
window by window over a ring of element buffers small enough to stay in L2. Every node
is still gathered once, summing its incident elements in element order, so the output
must equal the one-window assembly bit for bit, in both precisions, for the linear and
the material-point (J2) assembly with commits in between, and in a batch."""
import numpy as np
import pytest
import torch

from calculixpp_b200 import Plan
from calculixpp_b200 import meshgen as mg
from calculixpp_b200.assembly import Material
from tests.helpers import ALL_TYPES, box_model, to_np

pytestmark = pytest.mark.gpu

J2_STEEL = Material(210000.0, 0.3, ([0.0, 1.0], [250.0, 1250.0]), 0)


def _ring_budget(plan, tangent, window_elems):
    """Budget that gives windows of about `window_elems` elements for this plan."""
    m = plan.model.mesh
    n = m.conn.shape[1]
    nb = n * (n + 1) // 2
    blk = 80 if plan.precision == "fp64" else 48
    bpe = nb * blk + (24 * n if tangent else 0)
    conn = m.conn.astype(np.int64)
    order = np.argsort(conn.ravel(), kind="stable")
    elem = np.repeat(np.arange(m.n_elems), n)[order]
    node = conn.ravel()[order]
    first = np.full(m.n_nodes, m.n_elems)
    last = np.full(m.n_nodes, -1)
    np.minimum.at(first, node, elem)
    np.maximum.at(last, node, elem)
    span = int((last - first + 1).max())
    return (window_elems + span) * bpe


@pytest.mark.parametrize("etype", ALL_TYPES)
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_windowed_linear_equals_one_window(cuda, etype, precision):
    quad = etype in (mg.C3D20, mg.C3D20R, mg.C3D15, mg.C3D10)
    dims = (6, 4, 4) if quad else (12, 6, 5)
    model = box_model(etype, *dims, seed=etype)
    f = model.external_load_vector()
    one = Plan(model, precision)
    one.set_ring_bytes(-1)
    v1, r1 = (to_np(t).copy() for t in one.assemble_linear(f))
    assert one.windows()[0] == 1
    win = Plan(model, precision)
    win.set_ring_bytes(_ring_budget(win, False, 32))
    v2, r2 = (to_np(t).copy() for t in win.assemble_linear(f))
    nw, ring = win.windows()
    assert nw > 2 and ring < model.mesh.n_elems, (nw, ring)
    assert np.array_equal(v1, v2)
    assert np.array_equal(r1, r2)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_windowed_tangent_equals_one_window(cuda, precision):
    model = box_model(mg.C3D8, 12, 6, 5, jitter=0.08, seed=3, materials=[J2_STEEL], load=False)
    one = Plan(model, precision)
    one.set_ring_bytes(-1)
    win = Plan(model, precision)
    win.set_ring_bytes(_ring_budget(win, True, 32))
    x = model.mesh.coords
    for k in range(1, 4):
        u = np.zeros_like(x)
        u[:, 0] = 0.0015 * k * x[:, 0] * (0.3 + x[:, 2] / x[:, 2].max())
        u[:, 2] = -0.0008 * k * x[:, 0] ** 2 / x[:, 0].max()
        u = u.reshape(-1)
        a = [to_np(t).copy() for t in one.assemble_tangent(u)]
        b = [to_np(t).copy() for t in win.assemble_tangent(u)]
        for p, q in zip(a, b):
            assert np.array_equal(p, q), k
        assert torch.equal(one.state(committed=False), win.state(committed=False)), k
        one.commit()
        win.commit()
    nw, ring = win.windows(tangent=True)
    assert nw > 2 and ring < model.mesh.n_elems
    assert float(one.state()[:, 6].max()) > 0.0


def test_default_budget_is_one_window(cuda):
    model = box_model(mg.C3D8, 6, 4, 4)
    plan = Plan(model)
    plan.assemble_linear(model.external_load_vector())
    assert plan.windows() == (1, model.mesh.n_elems)
