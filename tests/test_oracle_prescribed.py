"""The oracle's prescribed displacements against the reference's closed forms
(crates/solidfem/tests/validation/prescribed.rs): an enforced stretch of a unit cube gives the
exact uniform stress E * stretch, the prescribed values come back exactly, and the free corner
contracts by -nu * stretch (CPU)."""
import numpy as np
import pytest

STEEL = (200000.0, 0.3)
STRETCH = 0.001
CUBE_POINTS = [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]]
CUBE_TETS = [[0, 1, 2, 6], [0, 2, 3, 6], [0, 3, 7, 6], [0, 7, 4, 6], [0, 4, 5, 6], [0, 5, 1, 6]]


def stretched(nodes):
    """The held components of a uniaxial stretch along x (prescribed.rs:40-60)."""
    out = []
    at = {tuple(p): i for i, p in enumerate(nodes.tolist())}
    for i, p in enumerate(nodes):
        if p[0] == 0.0:
            out.append((i, 0, 0.0))
        if p[0] == 1.0:
            out.append((i, 0, STRETCH))
    out += [(at[(0.0, 0.0, 0.0)], 1, 0.0), (at[(0.0, 0.0, 0.0)], 2, 0.0), (at[(0.0, 1.0, 0.0)], 2, 0.0)]
    return out


@pytest.mark.parametrize("multigrid", [False, True])
def test_oracle_stretched_cube(oracle, multigrid):
    mesh = oracle.Mesh.linear(np.array(CUBE_POINTS, dtype=np.float64), np.array(CUBE_TETS, dtype=np.uint32))
    nodes = mesh.nodes()
    opts = oracle.default_options(tolerance=1e-12, precision=oracle.DOUBLE,
                                  preconditioner=oracle.MULTIGRID if multigrid else oracle.JACOBI)
    st = oracle.Study(mesh, oracle.uniform(*STEEL), opts, [], prescribed=stretched(nodes))
    st.solve()
    d = st.displacements()
    assert np.all(d[nodes[:, 0] == 1.0, 0] == STRETCH)
    assert np.all(d[nodes[:, 0] == 0.0, 0] == 0.0)
    corner = int(np.flatnonzero(np.all(nodes == 1.0, axis=1))[0])
    assert abs(d[corner, 1] - (-STEEL[1] * STRETCH)) < 1e-6 * STRETCH
    st.recover()
    expected = STEEL[0] * STRETCH
    for p in st.point_stresses():
        assert abs(p.stress[0] - expected) < 1e-5 * expected
        for c in list(p.stress)[1:]:
            assert abs(c) < 1e-5 * expected
