"""Many oracle solves at once, in a spawned process pool.

TEST INFRASTRUCTURE ONLY: imported by tests/ and bench.py as the checker;
the product library never imports it.

Each work item names an RVE by plain numbers (mesh edge n, fibre radius,
materials), so worker processes import only the oracle (no CUDA context is
ever forked).  The solves are oracle.homogenize / unit_tangent /
fd_tangent at the oracle's tight tolerances (relative residual 1e-12),
which restate micro/src/homogenize.c:175-368 and :59-94.
"""
from __future__ import annotations

import multiprocessing as mp
import os

import numpy as np

RTOL, LIN_RTOL = 1e-12, 1e-13


def _mesh(n, radius):
    from . import oracle as O
    m = O.cube_mesh(int(n))
    return m, O.fiber_types(m, [1.0, 1.0], float(radius))


def homogenize(item):
    """item = (n, radius, (Em, Ef), (num, nuf), strains [k,6]) -> stress [k,6]."""
    from . import oracle as O
    n, radius, E, nu, strains = item
    m, et = _mesh(n, radius)
    _, st, _, _ = O.homogenize(m, et, tuple(E), tuple(nu), np.asarray(strains), rtol=RTOL,
                               lin_rtol=LIN_RTOL)
    return st


def unit_tangent(item):
    """item = (n, radius, (Em, Ef), (num, nuf)) -> C [6,6] from 6 unit strains."""
    from . import oracle as O
    n, radius, E, nu = item
    m, et = _mesh(n, radius)
    Cm, _ = O.unit_tangent(m, et, tuple(E), tuple(nu), rtol=RTOL, lin_rtol=LIN_RTOL)
    return Cm


def fd_tangent(item):
    """item = (n, radius, (Em, Ef), (num, nuf), eps [6]) -> (stress [6], C [6,6]),
    the finite-difference tangent of micro/src/homogenize.c:59-94."""
    from . import oracle as O
    n, radius, E, nu, eps = item
    m, et = _mesh(n, radius)
    Cm, s0 = O.fd_tangent(m, et, tuple(E), tuple(nu), np.asarray(eps, dtype=np.float64),
                          rtol=RTOL, lin_rtol=LIN_RTOL)
    return s0, Cm


def homogenize_periodic(item):
    """item = (n, radius, (Em, Ef), (num, nuf), strains [k,6]) -> stress [k,6]
    under periodic conditions (oracle/periodic.py, direct solve)."""
    from . import periodic as PER
    n, radius, E, nu, strains = item
    m, et = _mesh(n, radius)
    _, st, _ = PER.homogenize_periodic(m, et, tuple(E), tuple(nu), np.asarray(strains))
    return st


def run(fn, items, procs: int = 0):
    """[fn(item) for item in items], largest meshes first over a spawned pool
    of `procs` processes (0: every host core, at most len(items))."""
    items = list(items)
    procs = procs or min(len(items), os.cpu_count() or 1)
    if procs <= 1 or len(items) <= 1:
        return [fn(it) for it in items]
    order = sorted(range(len(items)), key=lambda i: -int(items[i][0]))
    with mp.get_context("spawn").Pool(procs) as pool:
        res = pool.map(fn, [items[i] for i in order], chunksize=1)
    out = [None] * len(items)
    for i, r in zip(order, res):
        out[i] = r
    return out
