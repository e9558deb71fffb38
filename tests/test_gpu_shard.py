"""Row-sharded assembly through the CUDA path: the shards of one model, assembled one
after another on one GPU (no rank waits on another), give owned rows that concatenate
to the single-plan K_ff, rhs and internal force bit for bit, in the linear and in the
J2 material-point assembly."""
import numpy as np
import pytest

from calculixpp_b200 import Plan
from calculixpp_b200 import meshgen as mg
from calculixpp_b200.assembly import Material
from calculixpp_b200.shard import (make_shard, node_row_weights, owned_elements, owned_nodal, owned_rows,
                                   partition_nodes, shard_state)
from tests.helpers import box_model, to_np

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("etype", [mg.C3D8, mg.C3D20, mg.C3D6])
def test_linear_shards(cuda, etype, precision):
    model = box_model(etype, 5, 3, 3, jitter=0.08, seed=etype)
    full = Plan(model, precision)
    v, r = (to_np(t) for t in full.assemble_linear(model.external_load_vector()))
    rp, ci = (to_np(t) for t in full.pattern())
    cuts = partition_nodes(node_row_weights(model), 3)
    got = []
    for k in range(3):
        sh = make_shard(model, cuts, k)
        p = Plan(sh.model, precision)
        lv, lr = (to_np(t) for t in p.assemble_linear(sh.model.external_load_vector()))
        lrp, lci = (to_np(t) for t in p.pattern())
        got.append(owned_rows(sh, lrp, lci, lv, lr))
        p.close()
    assert np.array_equal(np.concatenate([g[1] for g in got]), ci)
    assert np.array_equal(np.concatenate([g[2] for g in got]), v)
    assert np.array_equal(np.concatenate([g[3] for g in got]), r)
    assert sum(g[0][-1] for g in got) == rp[-1]
    full.close()


def test_tangent_shards_with_history(cuda):
    table = (np.array([0.0, 1.0]), np.array([250.0, 1250.0]))
    model = box_model(mg.C3D8, 6, 3, 3, jitter=0.05, seed=2, materials=[Material(210000.0, 0.3, table)],
                      load=False, prescribe=0.03)
    u = np.zeros(3 * model.mesh.n_nodes)
    u[0::3] = 0.03 * model.mesh.coords[:, 0] / 6.0 * (1.0 + 0.3 * model.mesh.coords[:, 2] / 3.0)
    full = Plan(model)
    committed = np.zeros((full.n_gauss, 13))
    v, fi, r = (to_np(t) for t in full.assemble_tangent(u))
    trial = to_np(full.state(committed=False))
    assert (trial[:, 6] > 0).mean() > 0.1
    cuts = partition_nodes(node_row_weights(model), 2)
    parts, f_parts = [], []
    for k in range(2):
        sh = make_shard(model, cuts, k)
        p = Plan(sh.model)
        p.set_state(shard_state(sh, committed, 8))
        lv, lfi, lr = (to_np(t) for t in p.assemble_tangent(u.reshape(-1, 3)[sh.nodes].reshape(-1)))
        lrp, lci = (to_np(t) for t in p.pattern())
        parts.append(owned_rows(sh, lrp, lci, lv, lr))
        f_parts.append(owned_nodal(sh, lfi))
        st = to_np(p.state(committed=False)).reshape(-1, 8, 13)
        own = owned_elements(sh)
        assert np.array_equal(st[own], trial.reshape(-1, 8, 13)[sh.elems[own]])
        p.close()
    assert np.array_equal(np.concatenate([q[2] for q in parts]), v)
    assert np.array_equal(np.concatenate([q[3] for q in parts]), r)
    assert np.array_equal(np.concatenate(f_parts), fi)
    full.close()
