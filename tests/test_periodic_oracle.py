"""The CPU periodic-conditions oracle (oracle/periodic.py) on its own:
<eps> = eps exactly, a homogeneous RVE gives D, the tangent is symmetric
and no stiffer than the affine-displacement tangent (Hill bounds)."""
import numpy as np

from oracle import oracle as O
from oracle import periodic as P

E, NU = (1e9, 2.5e10), (0.3, 0.2)


def test_periodic_oracle_properties():
    m = O.cube_mesh(5)
    et = O.fiber_types(m, [1, 1], 0.3)
    sa, st, u = P.homogenize_periodic(m, et, E, NU, np.eye(6))
    assert np.abs(sa - np.eye(6)).max() <= 1e-12
    Cp = st.T
    assert np.abs(Cp - Cp.T).max() <= 1e-12 * np.abs(Cp).max()
    _, sta, _, _ = O.homogenize(m, et, E, NU, np.eye(6), rtol=1e-12, lin_rtol=1e-13)
    dC = sta.T - Cp
    assert np.linalg.eigvalsh((dC + dC.T) / 2).min() >= -1e-6 * np.abs(Cp).max()
    # periodicity of the fluctuation: u(x + L) - u(x) = eps . L on opposite faces
    nx = m.nx
    U = u[0].reshape(nx, nx, nx, 3)  # [k][j][i][d]
    assert np.abs((U[:, :, -1, 0] - U[:, :, 0, 0]) - 1.0).max() <= 1e-12


def test_periodic_oracle_homogeneous_patch():
    m = O.cube_mesh(4)
    et = np.zeros(m.nelm, dtype=np.uint8)
    _, st, _ = P.homogenize_periodic(m, et, E, NU, np.eye(6))
    D = np.zeros(36)
    O.lib().orc_iso_D(3, E[0], NU[0], O.ptr(D))
    assert np.abs(st.T - D.reshape(6, 6)).max() <= 1e-12 * E[0]
