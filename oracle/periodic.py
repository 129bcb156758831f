"""CPU restatement of 3D periodic boundary conditions by master-slave
elimination (numpy + scipy).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker; the product
library never imports it.

The reference declares a master-slave periodic condition (BC_PER_MS,
micro/inc/micro.h:26) without implementing it, and implements the 2D
Lagrange-multiplier variant (micro/src/assembly.c:175-220 residual,
:272-354 Jacobian): corner displacements prescribed to eps.x and opposite
face nodes tied by u+ - u- = eps.dl.  This oracle states the same
conditions in 3D by elimination: u = eps.x + P w with the fluctuation w on
the periodic grid (node (i mod n, j mod n, k mod n)); every corner maps to
periodic node 0, whose w is fixed to 0 (the corners carry eps.x).  The
equations are P^T K P w = -P^T K (eps.x) on the free periodic dofs, solved
directly; averages use the oracle's own get_averages restatement.  No
reference vectors exist for this condition (parity unpinned): the checks
are this restatement, exact patch properties and the Hill bounds.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O


def _pieces(m, etype, E, nu):
    import scipy.sparse as sps

    _, Ke, _, _ = O.operators(m, E, nu)
    dofs = O.elem_dofs(m)
    vals = Ke[etype].reshape(len(etype), -1)
    rows = np.repeat(dofs, 24, axis=1).ravel()
    cols = np.tile(dofs, (1, 24)).ravel()
    K = sps.coo_matrix((vals.ravel(), (rows, cols)), shape=(m.ndof, m.ndof)).tocsr()
    node = np.arange(m.nn)
    i, j, k = node % m.nx, (node // m.nx) % m.ny, node // (m.nx * m.ny)
    nex, ney, nez = m.nx - 1, m.ny - 1, m.nz - 1
    per = (i % nex) + nex * ((j % ney) + ney * (k % nez))
    npd = 3 * nex * ney * nez
    r = (3 * node[:, None] + np.arange(3)).ravel()
    c = (3 * per[:, None] + np.arange(3)).ravel()
    P = sps.coo_matrix((np.ones(len(r)), (r, c)), shape=(m.ndof, npd)).tocsr()
    X = np.stack([i * m.hx, j * m.hy, k * m.hz], 1)
    return K, P, X, npd


def affine_field(X, strain) -> np.ndarray:
    """u = eps.x on every node, engineering shears halved (the reference's
    strain_x_coord, micro/src/homogenize.c:335-342, in 3D)."""
    e = np.asarray(strain, dtype=np.float64)
    u = np.empty((len(X), 3))
    u[:, 0] = e[0] * X[:, 0] + e[3] / 2 * X[:, 1] + e[5] / 2 * X[:, 2]
    u[:, 1] = e[3] / 2 * X[:, 0] + e[1] * X[:, 1] + e[4] / 2 * X[:, 2]
    u[:, 2] = e[5] / 2 * X[:, 0] + e[4] / 2 * X[:, 1] + e[2] * X[:, 2]
    return u.ravel()


def homogenize_periodic(m, etype, E, nu, strains):
    """(strain_ave [k,6], stress_ave [k,6], u [k,ndof]) for each strain."""
    import scipy.sparse.linalg as spl

    K, P, X, npd = _pieces(m, etype, E, nu)
    Kp = (P.T @ K @ P).tocsc()
    keep = np.arange(3, npd)  # periodic node 0 (every corner) fixed
    Kk = Kp[keep][:, keep].tocsc()
    lu = spl.splu(Kk)
    strains = np.atleast_2d(strains)
    sa, st, us = [], [], []
    for s in strains:
        ua = affine_field(X, s)
        f = -(P.T @ (K @ ua))
        w = np.zeros(npd)
        w[keep] = lu.solve(f[keep])
        u = ua + P @ w
        a, b = O.averages(m, etype, E, nu, u)
        sa.append(a)
        st.append(b)
        us.append(u)
    return np.array(sa), np.array(st), np.array(us)
