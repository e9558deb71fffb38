"""Thermal strain on the device (cxg_plan_set_thermal_strain).

Against the oracle (pinned bit-exact to the reference by test_oracle_thermal.py), with a
constant alpha and an alpha(T) table and temperatures applied on part of the nodes:
* cxg_thermal_strain_load = thermal_strain_load_vector within 1e-12 relative;
* the Gauss-point stress D (eps - eps_th), nodal strain / stress and reactions
  f_int - f_ext with f_int = K u - f_th within 1e-12;
* the linear assembly's rhs carries the thermal-strain load: equal within 1e-12 to the
  reference's own assemble_linear_static rhs; clearing the inputs restores the rhs.
"""
import numpy as np
import pytest

from calculixpp_b200 import Plan
from calculixpp_b200 import meshgen as mg
from tests.helpers import ALL_TYPES, rel_fro, to_np
from tests.test_oracle_thermal import _thermal_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("etype", ALL_TYPES)
def test_thermal_load_and_recovery(cuda, port, etype):
    model, m, mats, em, tables, trefs, T, applied, thermal = _thermal_case(etype, 40 + etype)
    plan = Plan(model)
    plan.set_thermal_strain(*thermal)
    f_o = port.thermal_strain_load(m, m.young, m.poisson, thermal)
    assert rel_fro(to_np(plan.thermal_strain_load()), f_o) <= 1e-12
    u = np.random.default_rng(etype + 9).uniform(-1e-3, 1e-3, 3 * m.n_nodes)
    sg = to_np(plan.recover_gauss_stress(u))
    assert rel_fro(sg.reshape(-1), port.recover_gauss_stress_th(m, m.young, m.poisson, thermal, u).reshape(-1)) <= 1e-12
    if etype == mg.C3D8R:
        return  # nodal field recovery is not provided for C3D8R
    f_ext = model.external_load_vector()
    st, ss, rf = (to_np(x) for x in plan.recover_fields(u, f_ext))
    so, sso, rfo = port.recover_fields_th(m, m.young, m.poisson, thermal, u, f_ext)
    assert rel_fro(st.reshape(-1), so.reshape(-1)) <= 1e-12
    assert rel_fro(ss.reshape(-1), sso.reshape(-1)) <= 1e-12
    assert rel_fro(rf.reshape(-1), rfo.reshape(-1)) <= 1e-12


@pytest.mark.parametrize("etype", [mg.C3D8, mg.C3D20, mg.C3D10, mg.C3D15])
def test_linear_rhs_matches_reference(cuda, ref, etype):
    model, m, mats, em, tables, trefs, T, applied, thermal = _thermal_case(etype, 70 + etype)
    rm = ref.model(m, mats, em, model.spc, model.cloads)
    rm.set_expansion(tables, trefs)
    on = np.flatnonzero(applied)
    rm.set_temperature(on, T[on])
    sys_ = rm.assemble_linear_static()
    plan = Plan(model)
    f_ext = model.external_load_vector()
    _, rhs0 = (to_np(x).copy() for x in plan.assemble_linear(f_ext))
    plan.set_thermal_strain(*thermal)
    _, rhs = (to_np(x).copy() for x in plan.assemble_linear(f_ext))
    assert rel_fro(rhs, sys_["rhs"]) <= 1e-12
    assert rel_fro(rhs - rhs0, rhs) > 1e-3  # the thermal load is a large part of the rhs
    plan.set_thermal_strain(None)
    _, rhs1 = (to_np(x).copy() for x in plan.assemble_linear(f_ext))
    assert np.array_equal(rhs1, rhs0)


def test_thermal_inputs_validated(cuda):
    model, m, mats, em, tables, trefs, T, applied, thermal = _thermal_case(mg.C3D8, 3)
    plan = Plan(model)
    with pytest.raises(ValueError):
        plan.set_thermal_strain(T, applied, thermal[2][:-1], thermal[3])
    plan.set_thermal_strain(None)
    assert np.abs(to_np(plan.thermal_strain_load())).max() == 0.0
