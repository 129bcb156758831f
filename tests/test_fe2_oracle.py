"""The CPU FE2 oracle (oracle/fe2.py) on its own: its element arithmetic is
the micro oracle's (pinned against the reference's fem.c), the Newton loop
converges in one step without strain clipping, and a homogeneous cantilever
bends as beam theory predicts."""
import numpy as np

from oracle import fe2 as F
from oracle import oracle as O


def iso_C(E, nu):
    D = np.zeros(36)
    O.lib().orc_iso_D(3, E, nu, O.ptr(D))
    return D.reshape(6, 6)


def test_macro_element_matches_micro_element_stiffness():
    n, length = (3, 2, 2), (1.5, 1.0, 1.0)
    m, B, w, dofs = F.box_ops(n, length)
    C = iso_C(2e9, 0.27)
    Ke = np.einsum("ghi,hk,gkj,g->ij", B, C, B, w)
    _, Ke_o, _, _ = O.operators(m, (2e9, 2e9), (0.27, 0.27))
    assert np.abs(Ke - Ke_o[0]).max() <= 1e-12 * np.abs(Ke_o[0]).max()


def test_newton_converges_in_one_step_without_clip():
    n, length = (6, 2, 2), (3.0, 1.0, 1.0)
    C = np.broadcast_to(iso_C(1e9, 0.3), (np.prod(n), 8, 6, 6)).copy()
    u, norms = F.fe2_cantilever(n, length, (0, 0, -1e5), C, newton_its=3, strain_clip=0.0)
    assert norms[1] <= 1e-9 * norms[0] and norms[2] <= 1e-9 * norms[0]


def test_homogeneous_cantilever_tip_deflection_near_beam_theory():
    n, length = (20, 4, 4), (10.0, 1.0, 1.0)
    E, nu, t = 1e9, 0.3, -1e4
    C = np.broadcast_to(iso_C(E, nu), (np.prod(n), 8, 6, 6)).copy()
    u, _ = F.fe2_cantilever(n, length, (0, 0, t), C, newton_its=1, strain_clip=0.0)
    m, _, _, _ = F.box_ops(n, length)
    face = np.array([(m.nx - 1) + j * m.nx + k * m.nx * m.ny for k in range(m.nz) for j in range(m.ny)])
    tip = u[3 * face + 2].mean()
    P = t * 1.0 * 1.0
    I = 1.0 / 12.0
    eb = P * 10.0 ** 3 / (3 * E * I)
    # trilinear hexa8 bending is too stiff on coarse meshes; beam theory is an
    # upper bound in magnitude and the mesh gets within 25% of it
    assert 0.75 * abs(eb) <= abs(tip) <= 1.02 * abs(eb)
    assert np.sign(tip) == np.sign(eb)
