"""Parity of the plain FP64 RVE path (sp_rve_*) against the oracle: element
stiffness bit-exact, ELL columns bit-exact with the reference's insertion
order, ELL values to rounding, displacements / stresses / tangent to the
1e-8 relative tolerance of the hot path."""
import numpy as np
import pytest

import madmax_b200 as mb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

E, NU = (1e9, 1e10), (0.3, 0.2)


def rel2(a, b):
    """Norm-wise relative difference ||a - b|| / ||b|| (a residual bound of
    1e-8 controls this, not the worst single entry)."""
    return np.linalg.norm(np.asarray(a) - b) / np.linalg.norm(b)


def oracle_ref(n, radius, strains, E=E, nu=NU):
    m = O.cube_mesh(n)
    et = O.fiber_types(m, [1, 1], radius)
    sa, st, u, stats = O.homogenize(m, et, E, nu, strains, want_u=True, rtol=1e-12,
                                    lin_rtol=1e-13)
    return m, et, sa, st, u


@pytest.mark.parametrize("n,radius", [(2, 0.3), (5, 0.25), (10, 0.25)])
def test_ke_and_ell_assembly(n, radius):
    r = mb.Rve(mb.rve_desc(n, radius, E, NU))
    m = O.cube_mesh(n)
    et = O.fiber_types(m, [1, 1], radius)
    assert np.array_equal(mb.classify(r.desc), et)
    assert r.nfiber == int(et.sum())
    _, Ke, _, _ = O.operators(m, E, NU)
    km, kf = r.ke()
    assert np.array_equal(km, Ke[0]) and np.array_equal(kf, Ke[1])
    cols, vals = r.ell()
    A = O.assemble(m, et, E, NU, symmetric_bc=True)
    assert np.array_equal(cols, A.cols)
    assert np.array_equal(cols, mb.ell_pattern(n))
    scale = np.abs(A.vals).max(axis=1, keepdims=True)
    assert (np.abs(vals - A.vals) <= 4e-16 * 8 * scale).all()


def test_cfg1_stress_matches_oracle():
    """10x10x10 RVE, fiber r = 0.25, eps = (1e-3, 0, ...)."""
    eps = [[1e-3, 0, 0, 0, 0, 0]]
    m, et, sa, st, u = oracle_ref(10, 0.25, eps)
    r = mb.Rve(mb.rve_desc(10, 0.25, E, NU))
    gsa, gst, gu, info = r.homogenize(eps, rtol=1e-8, want_u=True)
    assert info.status == 0 and info.relres <= 1e-8
    assert np.abs(gst - st).max() <= 1e-8 * np.abs(st).max()
    assert np.abs(gsa - sa).max() <= 1e-8 * np.abs(sa).max()
    assert rel2(gu, u) <= 1e-8


@pytest.mark.parametrize("nrhs", [1, 3, 6, 7, 8])
def test_multi_rhs_matches_oracle(nrhs):
    rng = np.random.default_rng(nrhs)
    eps = rng.normal(0, 1e-3, size=(nrhs, 6))
    m, et, sa, st, u = oracle_ref(6, 0.3, eps, E=(2e9, 1e11), nu=(0.25, 0.33))
    r = mb.Rve(mb.rve_desc(6, 0.3, (2e9, 1e11), (0.25, 0.33)))
    gsa, gst, gu, info = r.homogenize(eps, rtol=1e-8, want_u=True)
    assert info.status == 0
    for k in range(nrhs):
        assert np.abs(gst[k] - st[k]).max() <= 1e-8 * np.abs(st[k]).max()
        assert rel2(gu[k], u[k]) <= 1e-8


def test_tangent_matches_oracle():
    m = O.cube_mesh(8)
    et = O.fiber_types(m, [1, 1], 0.3)
    C6, _ = O.unit_tangent(m, et, E, NU, rtol=1e-12, lin_rtol=1e-13)
    r = mb.Rve(mb.rve_desc(8, 0.3, E, NU))
    G, info = r.tangent(rtol=1e-8)
    assert info.status == 0
    assert np.abs(G - C6).max() <= 1e-8 * np.abs(C6).max()
    # major symmetry of the homogenized tangent (symmetric operator)
    assert np.abs(G - G.T).max() <= 1e-7 * np.abs(G).max()


def test_non_cubic_mesh_and_offset_fiber():
    d = mb.rve_desc((4, 6, 3), 0.35, E, NU, length=(1.0, 1.5, 0.75), desv=(0.1, -0.2))
    m = O.mesh(3, [5, 7, 4], [1.0, 1.5, 0.75])
    et = O.fiber_types(m, [1.0, 1.5], 0.35, desv=(0.1, -0.2))
    r = mb.Rve(d)
    assert np.array_equal(mb.classify(d), et)
    eps = [[0, 1e-3, 0, 0, 0, 2e-3]]
    sa, st, u, _ = O.homogenize(m, et, E, NU, eps, want_u=True, rtol=1e-12, lin_rtol=1e-13)
    gsa, gst, gu, info = r.homogenize(eps, want_u=True)
    assert info.status == 0
    assert np.abs(gst - st).max() <= 1e-8 * np.abs(st).max()


def test_element_fields_and_vtu_match_oracle(tmp_path):
    """Per-element strain/stress (get_elem_properties, micro/src/homogenize.c:
    370-395) of the second load case against the oracle's solution, their
    volume average against the homogenized stress, and the VTU piece."""
    import xml.etree.ElementTree as ET
    n, rad, E, nu = 5, 0.3, (1e9, 2e10), (0.3, 0.2)
    d = mb.rve_desc(n, rad, E, nu)
    r = mb.Rve(d)
    strains = np.array([[1e-3, 0, 0, 0, 0, 0], [2e-4, -1e-4, 3e-4, 1e-4, 0.0, -2e-4]])
    _, st, _, info = r.homogenize(strains, rtol=1e-10)
    se, ss, u, res = r.fields(1)
    m = O.cube_mesh(n)
    et = O.fiber_types(m, [1, 1], rad)
    _, sto, uo, _ = O.homogenize(m, et, E, nu, strains, want_u=True, rtol=1e-12, lin_rtol=1e-13)
    D, _, bmat, wp = O.operators(m, E, nu)
    B = bmat.reshape(6, 24, 8)
    dofs = O.elem_dofs(m)
    eps_o = np.einsum("vig,ei,g->ev", B, uo[1][dofs], wp) / m.vol_elm
    sig_o = np.einsum("evw,ew->ev", D[et], eps_o)
    assert np.abs(u - uo[1]).max() <= 1e-8 * np.abs(uo[1]).max()
    assert np.abs(se - eps_o).max() <= 1e-8 * np.abs(eps_o).max()
    assert np.abs(ss - sig_o).max() <= 1e-8 * np.abs(sig_o).max()
    assert np.abs(ss.mean(0) - st[1]).max() <= 1e-10 * np.abs(st[1]).max()
    base = str(tmp_path / "micro")
    r.write_vtu(base, 1)
    v = ET.parse(base + "_0.vtu").getroot()
    arr = {da.get("Name"): np.array(da.text.split(), dtype=float) for da in v.iter("DataArray")}
    assert np.allclose(arr["displ"], u, rtol=1e-8, atol=1e-30)
    assert np.allclose(arr["stress"].reshape(-1, 6), ss, rtol=1e-8, atol=1e-30)
    assert (arr["elem_type"] == et).all()
    with pytest.raises(mb.SputnikError):
        r.fields(2)
    r.close()
