"""The C ABI library loads and exports exactly what include/cxg.h declares; entry
points that need no GPU behave; plan creation without a GPU fails with a status."""
import ctypes as C
import os
import re

import pytest

from calculixpp_b200 import _lib
from calculixpp_b200 import meshgen as mg

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "cxg.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"CXG_API\s+[\w\s\*]+?\b(cxg_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name


def test_python_binding_covers_header():
    assert set(declared()) == set(_lib.SIGNATURES)


def test_version_and_tables():
    lib = _lib.load()
    text = open(HEADER).read()
    version = int(re.search(r"#define CXG_ABI_VERSION (\d+)", text).group(1))
    assert lib.cxg_abi_version() == version
    for t in mg.NODES:
        assert lib.cxg_nodes_per_element(t) == mg.NODES[t]
        assert lib.cxg_gauss_points_per_element(t) == mg.NGP[t]
    assert lib.cxg_nodes_per_element(8) == 0  # not an element type code


def test_plan_create_without_gpu_reports_status():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from calculixpp_b200.assembly import Material, Model, Plan
    m = mg.box_mesh(mg.C3D8, 1, 1, 1)
    with pytest.raises(_lib.CxgError) as exc:
        Plan(Model(m, [Material(210000.0, 0.3)]))
    assert exc.value.code == _lib.CXG_ERR_NO_GPU


def test_invalid_arguments_rejected_before_device_use():
    lib = _lib.load()
    out = C.c_void_p()
    rc = lib.cxg_plan_create(None, None, 0, C.byref(out))
    assert rc == _lib.CXG_ERR_INVALID_ARGUMENT
    assert lib.cxg_last_error()
    rc = lib.cxg_element_stiffness(8, 1, None, None, None, 0, None, None)  # no such element type
    assert rc == _lib.CXG_ERR_UNSUPPORTED
