"""CPU restatement of the FE2 macro Newton loop (numpy + scipy).

TEST INFRASTRUCTURE ONLY: imported by tests/ and bench.py as the checker;
the product library never imports it.

It follows the reference's macro driver:
  - Newton loop: macro/src/main.c:202-256 (residual norm checked before the
    Jacobian is assembled, x += dx);
  - residual b = -sum_e sum_gp B^T sigma w with Dirichlet rows zeroed:
    macro/src/assembly.c:5-84 (here with the consistent nodal forces of a
    uniform traction added: b = f_ext - f_int);
  - Jacobian sum_e sum_gp B^T C B w, Dirichlet rows and columns set to the
    identity: macro/src/assembly.c:165-222 (MatZeroRowsColumns, :208-214);
  - Gauss-point strain B u_e with components below 1e-6 set to zero:
    macro/src/assembly.c:305-322;
  - hexa8 B matrices and Gauss weights from the oracle's restatement of
    src/fem.c:309-405 and micro/src/init.c:40-51 (oracle.c), so the element
    arithmetic is the one pinned against the reference's own fem.c.
The linear systems are solved directly (scipy spsolve), so the oracle's
Newton iterates carry no Krylov tolerance.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O


def box_ops(n, length):
    """(mesh, B[8 gp][6][24], w[8], element dofs [nelm][24])."""
    m = O.mesh(3, [n[0] + 1, n[1] + 1, n[2] + 1], list(length))
    ngp, nc = m.ngp, m.npe * m.dim
    dsh = np.zeros(nc * ngp)
    wp = np.zeros(ngp)
    O.lib().orc_struct_dsh(O.C.byref(m), O.ptr(dsh), O.ptr(wp))
    bmat = np.zeros(m.nvoi * nc * ngp)
    O.lib().orc_bmat(O.C.byref(m), O.ptr(dsh), O.ptr(bmat))
    B = bmat.reshape(m.nvoi, nc, ngp).transpose(2, 0, 1).copy()
    return m, B, wp, O.elem_dofs(m)


def traction_forces(m, traction) -> np.ndarray:
    """Consistent nodal forces of a uniform traction on the face x = lx."""
    f = np.zeros(m.ndof)
    for k in range(m.nz):
        for j in range(m.ny):
            cy = 1 if j in (0, m.ny - 1) else 2
            cz = 1 if k in (0, m.nz - 1) else 2
            node = (m.nx - 1) + j * m.nx + k * m.nx * m.ny
            f[3 * node:3 * node + 3] = np.asarray(traction) * (m.hy * m.hz * cy * cz / 4.0)
    return f


def clamped_dofs(m) -> np.ndarray:
    nodes = np.arange(m.nn)
    fixed = nodes[nodes % m.nx == 0]
    return (3 * fixed[:, None] + np.arange(3)).ravel()


def fe2_cantilever(n, length, traction, C_gp, newton_its=5, strain_clip=1e-6, newton_tol=0.0):
    """Macro Newton loop with a fixed tangent per Gauss point (linear micro:
    sigma = C eps).  C_gp: [nelm, 8, 6, 6].  Returns (u, [||b|| per
    iteration])."""
    import scipy.sparse as sps
    import scipy.sparse.linalg as spl

    m, B, w, dofs = box_ops(n, length)
    fext = traction_forces(m, traction)
    fixed = clamped_dofs(m)
    free = np.ones(m.ndof, bool)
    free[fixed] = False
    u = np.zeros(m.ndof)
    # Jacobian (the same every iteration for a linear micro response)
    Ke = np.einsum("ghi,eghk,gkj,g->eij", B, C_gp, B, w)
    rows = np.repeat(dofs, 24, axis=1).ravel()
    cols = np.tile(dofs, (1, 24)).ravel()
    K = sps.coo_matrix((Ke.ravel(), (rows, cols)), shape=(m.ndof, m.ndof)).tocsr()
    D = sps.diags(free.astype(float))
    K = (D @ K @ D + sps.diags((~free).astype(float))).tocsc()
    norms = []
    for _ in range(newton_its):
        ue = u[dofs]
        eps = np.einsum("gvi,ei->egv", B, ue)
        eps[np.abs(eps) < strain_clip] = 0.0
        sig = np.einsum("egjk,egk->egj", C_gp, eps)
        fe = np.einsum("gvi,egv,g->ei", B, sig, w)
        fint = np.zeros(m.ndof)
        np.add.at(fint, dofs.ravel(), fe.ravel())
        b = fext - fint
        b[fixed] = 0.0
        norms.append(float(np.linalg.norm(b)))
        if norms[-1] <= newton_tol:
            break
        u = u + spl.spsolve(K, b)
    return u, norms
