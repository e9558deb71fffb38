"""The oracle's ctypes layer: every entry point carries its declared signature, handles
keep their full pointer width, and a failing call raises OracleError with the library's
message. A handle returned as a C int would be cut to 32 bits and only work while the
host heap stays below 2 GiB."""
import ctypes as C

import numpy as np
import pytest

from calculixpp_b200 import meshgen as mg
from oracle.oracle import PORT_SIGS, REF_SIGS, OracleError, make_material
from tests.helpers import unit_element

PORT_HANDLES = ("assemble_linear", "assemble_tangent", "assemble_scalar", "assemble_conduction")
REF_HANDLES = ("model_create", "assemble_linear_static", "mp_create", "assemble_material_tangent",
               "assemble_mass", "assemble_geometric", "assemble_conduction")


def _check_sigs(lib, sigs, handles):
    for name in handles:
        assert sigs[name][0] is C.c_void_p, name
    for name, (res, args) in sigs.items():
        f = lib._fn(name)
        assert f.restype is res, name
        assert list(f.argtypes) == list(args), name
        # the configured object is the one every later lookup returns
        assert lib._fn(name) is f
    assert lib._fn("last_error").restype is C.c_char_p


def test_port_signatures(port):
    _check_sigs(port, PORT_SIGS, PORT_HANDLES)


def test_ref_signatures(ref):
    _check_sigs(ref, REF_SIGS, REF_HANDLES)


def _inverted(etype):
    x = unit_element(etype)
    x[:, 2] *= -1.0  # mirror: every Jacobian determinant is negative
    return x


@pytest.mark.parametrize("which", ["port", "ref"])
def test_failing_call_raises_with_message(request, which):
    lib = request.getfixturevalue(which)
    with pytest.raises(OracleError, match="non-positive element Jacobian"):
        lib.element_stiffness(mg.C3D8, _inverted(mg.C3D8), 210000.0, 0.3)


def test_port_null_system_raises_with_message(port):
    m = mg.box_mesh(mg.C3D8, 2, 1, 1, 2.0, 1.0, 1.0)
    m.coords[:, 2] *= -1.0
    dof_eq = np.arange(3 * m.n_nodes, dtype=np.int32)
    with pytest.raises(OracleError, match="non-positive element Jacobian"):
        port.assemble_linear(m, [make_material(210000.0, 0.3)], None, dof_eq,
                             np.zeros(3 * m.n_nodes), 3 * m.n_nodes)


def test_ref_handles_round_trip(ref):
    """A model handle comes back as a full-width integer and survives create, assemble,
    material points and free."""
    m = mg.box_mesh(mg.C3D8, 2, 1, 1, 2.0, 1.0, 1.0)
    sn, sc, sv = mg.clamp_face_spc(m, 0, 0.0)
    rm = ref.model(m, [make_material(210000.0, 0.3)], spc=(sn, sc, sv))
    assert isinstance(rm.h, int) and rm.h > 0
    sys_ = rm.assemble_linear_static()
    assert sys_["n_free"] == 3 * m.n_nodes - sn.size
    mp = rm.material_points()
    assert isinstance(mp, int) and mp > 0
    assert rm.state().size == 13 * m.n_elems * mg.NGP[mg.C3D8]


def test_adapter_library_loads_with_its_signatures(ref):
    """The C++ adapter's test library (the product adapter compiled against the
    reference headers) loads without a GPU and exports every declared entry point."""
    from oracle.oracle import ADAPTER_SIGS, RefCuda
    if not RefCuda.available():
        pytest.skip("adapter library not built here")
    lib = RefCuda()
    _check_sigs(lib, ADAPTER_SIGS, ("assembler_create",))
