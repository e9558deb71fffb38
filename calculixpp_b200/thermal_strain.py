"""Host side of the thermal-strain inputs (*EXPANSION with an applied temperature field).

The reference evaluates, per element with an expansion (Material::expansion), the nodal
temperature change te_k = T_k - t_ref at the nodes with an applied temperature (0
elsewhere) and the expansion coefficient alpha(T) of the material's table at the element's
mean temperature, the nodes without an applied temperature counting as t_ref
(element_temp_change / element_alpha, src/fem/stress.cpp:76-105; the same in
thermal_strain_load_vector, src/fem/loads.cpp:531-550). The device kernels take the
per-node temperatures and the per-element alpha and t_ref that `thermal_strain_inputs`
returns.
"""
from __future__ import annotations

import numpy as np


def table_at(values, temps, T):
    """PropertyTable::at (include/calculixpp/core/material.hpp:100-109): piecewise-linear
    interpolation in T, clamped outside the table; a one-row table is constant."""
    v = [float(x) for x in values]
    t = [float(x) for x in temps]
    if not v:
        return 0.0
    if len(v) == 1 or T <= t[0]:
        return v[0]
    if T >= t[-1]:
        return v[-1]
    i = 1
    while i < len(t) and T > t[i]:
        i += 1
    t0, t1 = t[i - 1], t[i]
    w = 0.0 if t1 == t0 else (T - t0) / (t1 - t0)
    return v[i - 1] + w * (v[i] - v[i - 1])


def thermal_strain_inputs(conn, elem_mat, expansion, node_temp, node_applied=None):
    """(node_temp[N], node_applied[N] uint8, elem_alpha[E], elem_tref[E]) for the device.

    conn: (E, n) node indices; elem_mat: (E,) material index; expansion[k]: None or
    (alpha values, alpha temperatures, t_ref) of material k; node_temp: (N,) applied
    temperatures (ignored where node_applied is 0); node_applied: (N,) 0/1, None = all.
    Elements without an expansion get alpha 0."""
    conn = np.asarray(conn)
    E, n = conn.shape
    T = np.asarray(node_temp, dtype=np.float64)
    applied = np.ones(T.size, np.uint8) if node_applied is None else np.asarray(node_applied, dtype=np.uint8)
    elem_mat = np.asarray(elem_mat)
    alpha = np.zeros(E)
    tref = np.zeros(E)
    for k, ex in enumerate(expansion):
        if ex is None or len(ex[0]) == 0:
            continue
        sel = np.flatnonzero(elem_mat == k)
        if sel.size == 0:
            continue
        t_ref = float(ex[2])
        tref[sel] = t_ref
        # element mean temperature, summed node by node in element order
        tsum = np.zeros(sel.size)
        for j in range(n):
            nodes = conn[sel, j]
            tsum += np.where(applied[nodes] != 0, T[nodes], t_ref)
        mean = tsum / float(n)
        if len(ex[0]) == 1:
            alpha[sel] = float(ex[0][0])
        else:
            alpha[sel] = [table_at(ex[0], ex[1], m) for m in mean]
    return T, applied, alpha, tref
