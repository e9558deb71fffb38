"""ComputeBackend::solve_sparse on the device (include/calculixpp/compute/backend.hpp:51-56).

The reference's CPU backend converts COO triplets to CSR and calls a sparse direct solve
or IC0-preconditioned CG (src/compute/cpu_backend.cpp:24-72). `solve_sparse` takes the
same arguments and runs cxg_solve_sparse: the COO-to-CSR reduction (duplicates summed),
the factorisation and the iterations all on the device.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

SOLVERS = {"direct": _lib.SOLVER_DIRECT, "cg": _lib.SOLVER_IC0_CG, "cg_jacobi": _lib.SOLVER_CG}


def solve_sparse(rows, cols, vals, n, rhs, solver="direct", rtol=1e-10, max_iter=None):
    """x with A x = rhs for the n x n SPD matrix A given by COO triplets (duplicates summed).

    solver: "direct" (sparse Cholesky, the reference's default), "cg" (IC0-preconditioned
    CG, the reference's CG kind) or "cg_jacobi" (diagonal preconditioner). Raises CxgError
    (CXG_ERR_NOT_CONVERGED) when a CG kind misses rtol within max_iter, as the reference
    throws. Returns (x, iterations, relative residual)."""
    lib = _lib.load()
    r = np.ascontiguousarray(rows, dtype=np.int32)
    c = np.ascontiguousarray(cols, dtype=np.int32)
    v = np.ascontiguousarray(vals, dtype=np.float64)
    b = np.ascontiguousarray(rhs, dtype=np.float64)
    if not (r.size == c.size == v.size) or b.size != n:
        raise ValueError("solve_sparse: inconsistent COO / rhs sizes")
    x = np.zeros(n)
    it = C.c_int32(0)
    rel = C.c_double(0.0)
    mi = max(1000, 10 * n) if max_iter is None else int(max_iter)
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)
    _lib.check(lib.cxg_solve_sparse(n, v.size, ptr(r), ptr(c), ptr(v), ptr(b), ptr(x), SOLVERS[solver], rtol, mi,
                                    C.byref(it), C.byref(rel)))
    return x, it.value, rel.value
