"""cxg_element_tangent_force_noalloc: the element tangent/force entry point for callers
that cannot allocate device memory (code running inside another framework's memory
pool or a caller-managed arena, where cudaMalloc/cudaFree are off limits). Its scratch
lives in a fixed device buffer of the library, so it must give the same results as
cxg_element_tangent_force, call after call, with no state leaking from one call into
the next. Compared through the C ABI on two consecutive calls per element family and
precision, at the tolerances of the element tests (1e-12 relative on K_e and f_e in
FP64, 2e-5 in mixed precision; history 1e-10); both entry points run the same kernel,
so in practice the results agree bit for bit. Also covered: a batch of exactly
CXG_NOALLOC_MAX_GAUSS_POINTS points, and an empty batch."""
import ctypes as C

import numpy as np
import pytest
import torch

from calculixpp_b200 import _lib
from calculixpp_b200 import meshgen as mg
from calculixpp_b200.assembly import Material, _c_material
from tests.helpers import ISO_TABLE, distorted_elements, rel_fro

pytestmark = pytest.mark.gpu

MAT = Material(210000.0, 0.3, ISO_TABLE, 0)
LIMIT = 8192  # CXG_NOALLOC_MAX_GAUSS_POINTS (include/cxg.h)
TOL = {"fp64": 1e-12, "mixed": 2e-5}


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _run(name, etype, X, U, committed, precision="fp64"):
    lib = _lib.load()
    dev = torch.device("cuda")
    B, n, ngp = X.shape[0], mg.NODES[etype], mg.NGP[etype]
    nd = 3 * n
    x = torch.as_tensor(X, device=dev).contiguous()
    u = torch.as_tensor(U, device=dev).contiguous()
    sc = torch.as_tensor(committed, device=dev).contiguous()
    st = torch.full((B, ngp, 13), float("nan"), dtype=torch.float64, device=dev)
    Ke = torch.full((B, nd, nd), float("nan"), dtype=torch.float64, device=dev)
    fe = torch.full((B, nd), float("nan"), dtype=torch.float64, device=dev)
    keep = []
    cm = _c_material(MAT, keep)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    prec = _lib.MIXED if precision == "mixed" else _lib.FP64
    _lib.check(getattr(lib, name)(etype, B, _ptr(x), _ptr(u), C.byref(cm), _ptr(sc), _ptr(st), prec,
                                  _ptr(Ke), _ptr(fe), stream))
    torch.cuda.synchronize()
    return Ke.cpu().numpy(), fe.cpu().numpy(), st.cpu().numpy()


def _compare(etype, count, precision, seed):
    rng = np.random.default_rng(seed)
    X = distorted_elements(etype, count, seed=seed)
    G = rng.uniform(-0.012, 0.012, (count, 3, 3))
    U = np.einsum("bij,bkj->bki", G, X)
    committed = np.zeros((count, mg.NGP[etype], 13))
    tol = TOL[precision]
    for call in range(2):  # two consecutive calls: the second starts from the first's history
        Uk = U * (0.5 if call == 0 else 1.0)
        K0, f0, s0 = _run("cxg_element_tangent_force", etype, X, Uk, committed, precision)
        K1, f1, s1 = _run("cxg_element_tangent_force_noalloc", etype, X, Uk, committed, precision)
        assert rel_fro(K1, K0) <= tol, call
        assert rel_fro(f1, f0) <= tol, call
        assert np.all(np.abs(s1 - s0) <= 1e-10 * np.maximum(1.0, np.abs(s0))), call
        committed = s0
    assert np.any(committed[:, :, 6] > 0.0)  # the plastic branch was exercised


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("etype,count", [(mg.C3D8, 300), (mg.C3D20, 120), (mg.C3D8R, 64)])
def test_noalloc_matches_allocating_entry_point(cuda, etype, count, precision):
    _compare(etype, count, precision, seed=etype)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_at_exactly_the_limit(cuda, precision):
    """1024 C3D8 elements x 8 points fill the scratch exactly."""
    _compare(mg.C3D8, LIMIT // mg.NGP[mg.C3D8], precision, seed=41)


def test_noalloc_empty_batch(cuda):
    lib = _lib.load()
    keep = []
    cm = _c_material(MAT, keep)
    dev = torch.device("cuda")
    x = torch.zeros(8, dtype=torch.float64, device=dev)
    rc = lib.cxg_element_tangent_force_noalloc(mg.C3D8, 0, _ptr(x), _ptr(x), C.byref(cm), None, None,
                                               _lib.FP64, _ptr(x), _ptr(x), None)
    assert rc == _lib.CXG_OK


def test_noalloc_rejects_batches_beyond_its_scratch(cuda):
    lib = _lib.load()
    n_elems = LIMIT // mg.NGP[mg.C3D20] + 1
    dev = torch.device("cuda")
    x = torch.zeros(n_elems * 60, dtype=torch.float64, device=dev)
    keep = []
    cm = _c_material(MAT, keep)
    rc = lib.cxg_element_tangent_force_noalloc(mg.C3D20, n_elems, _ptr(x), _ptr(x), C.byref(cm), None, None,
                                               _lib.FP64, _ptr(x), _ptr(x), None)
    assert rc == _lib.CXG_ERR_INVALID_ARGUMENT
    assert b"exceeds the no-allocation limit" in lib.cxg_last_error()


def test_noalloc_rejects_host_arrays(cuda):
    lib = _lib.load()
    X = distorted_elements(mg.C3D8, 2, seed=1)
    keep = []
    cm = _c_material(MAT, keep)
    rc = lib.cxg_element_tangent_force_noalloc(mg.C3D8, 2, X.ctypes.data_as(C.c_void_p), X.ctypes.data_as(C.c_void_p),
                                               C.byref(cm), None, None, _lib.FP64, X.ctypes.data_as(C.c_void_p),
                                               X.ctypes.data_as(C.c_void_p), None)
    assert rc == _lib.CXG_ERR_INVALID_ARGUMENT
    assert b"device memory" in lib.cxg_last_error()
