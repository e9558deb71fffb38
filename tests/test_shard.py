"""Row-sharded assembly (calculixpp_b200.shard), host logic on the CPU.

The shards' owned rows, assembled by the oracle's C restatement of the reference
assembly, concatenate to the oracle's global K_ff and rhs bit for bit; the partition
covers every node once and balances the row non-zeros; two gloo ranks build their
shards independently and agree with the global system through an all-gather of
row ranges and checksums (no collective touches the data path itself)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from calculixpp_b200 import meshgen as mg
from calculixpp_b200.shard import make_shard, node_row_weights, owned_elements, owned_rows, partition_nodes
from tests.helpers import box_model, per_element_materials

CASES = [(mg.C3D8, (6, 3, 3)), (mg.C3D20, (3, 2, 2)), (mg.C3D15, (3, 2, 2)), (mg.C3D8R, (5, 2, 2))]


def oracle_system(port, model):
    mats, em = per_element_materials(model)
    dof_eq, pre, nf = model.dof_map()
    return port.assemble_linear(model.mesh, mats, em, dof_eq, pre, nf, model.external_load_vector())


@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_partition_covers_and_balances(world):
    model = box_model(mg.C3D8, 8, 4, 4, seed=1)
    w = node_row_weights(model)
    cuts = partition_nodes(w, world)
    assert cuts[0] == 0 and cuts[-1] == model.mesh.n_nodes and np.all(np.diff(cuts) > 0)
    loads = np.array([w[cuts[r]:cuts[r + 1]].sum() for r in range(world)])
    assert loads.max() <= loads.sum() / world + w.max() + 1


@pytest.mark.parametrize("etype,dims", CASES)
@pytest.mark.parametrize("world", [2, 3])
def test_owned_rows_concatenate_to_global_system(port, etype, dims, world):
    model = box_model(etype, *dims, jitter=0.08, seed=etype)
    model.mesh.young = model.mesh.young * np.random.default_rng(etype).uniform(0.5, 1.5, model.mesh.n_elems)
    rp, ci, v, rhs = oracle_system(port, model)
    cuts = partition_nodes(node_row_weights(model), world)
    parts = []
    owners = np.zeros(model.mesh.n_elems, dtype=int)
    for r in range(world):
        sh = make_shard(model, cuts, r)
        owners[sh.elems[owned_elements(sh)]] += 1
        lrp, lci, lv, lrhs = oracle_system(port, sh.model)
        parts.append((sh, owned_rows(sh, lrp, lci, lv, lrhs)))
    assert np.all(owners == 1)  # every element's history has exactly one owner
    assert [p[0].row0 for p in parts] == list(np.cumsum([0] + [p[0].n_rows for p in parts[:-1]]))
    g_rp = np.concatenate([[0]] + [p[1][0][1:] + sum(q[1][0][-1] for q in parts[:i]) for i, p in enumerate(parts)])
    assert np.array_equal(g_rp, rp)
    assert np.array_equal(np.concatenate([p[1][1] for p in parts]), ci)
    assert np.array_equal(np.concatenate([p[1][2] for p in parts]), v)
    assert np.array_equal(np.concatenate([p[1][3] for p in parts]), rhs)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port_no, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port_no)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle.oracle import Port
        port = Port()
        model = box_model(mg.C3D20, 4, 2, 2, jitter=0.08, seed=3)
        cuts = partition_nodes(node_row_weights(model), world)
        sh = make_shard(model, cuts, rank)
        lrp, lci, lv, lrhs = oracle_system(port, sh.model)
        orp, oci, ov, orhs = owned_rows(sh, lrp, lci, lv, lrhs)
        mine = torch.tensor([sh.row0, sh.n_rows, ov.size, float(ov.sum()), float(np.abs(ov).sum()),
                             float(orhs.sum()), float(oci.astype(np.float64).sum())], dtype=torch.float64)
        allv = [torch.zeros_like(mine) for _ in range(world)]
        dist.all_gather(allv, mine)
        if rank == 0:
            rp, ci, v, rhs = oracle_system(port, model)
            a = torch.stack(allv).numpy()
            ok = (a[0, 0] == 0 and np.all(a[1:, 0] == np.cumsum(a[:-1, 1])) and a[:, 1].sum() == rhs.size
                  and a[:, 2].sum() == v.size and np.isclose(a[:, 3].sum(), v.sum(), rtol=1e-12, atol=1e-6)
                  and np.isclose(a[:, 4].sum(), np.abs(v).sum(), rtol=1e-12)
                  and np.isclose(a[:, 5].sum(), rhs.sum(), rtol=1e-12, atol=1e-9)
                  and a[:, 6].sum() == ci.astype(np.float64).sum())
            out.put(bool(ok))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_build_shards_independently():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port_no = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port_no, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=5) is True
