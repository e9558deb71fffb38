"""Host-side pieces of bench.py that run without a GPU: the CSR pattern the CPU
baseline's scatter uses equals the oracle's assembled pattern (config-1 cantilever,
which has no exact-zero entries, so the topological and the value pattern agree)."""
import numpy as np

import bench
from calculixpp_b200 import meshgen as mg
from tests.helpers import per_element_materials
from calculixpp_b200.assembly import Material, Model


def test_host_pattern_matches_oracle(port):
    cfg = mg.cantilever_c3d8_config1()
    m, tip = cfg["mesh"], cfg["tip"]
    model = Model(m, [Material(210000.0, 0.3)], None, cfg["spc"],
                  (tip, np.full(tip.size, 2), np.full(tip.size, -1000.0 / tip.size)))
    dof_eq, pre, nf = model.dof_map()
    rp, ci = bench.host_pattern(m, dof_eq)
    mats, em = per_element_materials(model)
    orp, oci, _, _ = port.assemble_linear(m, mats, em, dof_eq, pre, nf)
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
