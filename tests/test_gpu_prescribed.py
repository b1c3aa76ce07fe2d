"""Prescribed displacements on the device (needs a B200): the reference's closed forms for a
stretched cube (crates/solidfem/tests/validation/prescribed.rs), and a clamped, loaded cantilever
with prescribed components whose eliminated operator and right-hand side equal the oracle's to the
bit and whose answer matches the oracle's."""
import numpy as np
import pytest

import solidfem_b200 as sf
from tests.helpers import ON_PLANE
from tests.test_oracle_prescribed import CUBE_POINTS, CUBE_TETS, STEEL, STRETCH, stretched

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pre", ["jacobi", "double", "mixed"])
def test_stretched_cube_closed_forms(pre):
    mesh = sf.Mesh.from_linear(np.array(CUBE_POINTS, dtype=np.float64), np.array(CUBE_TETS, dtype=np.uint32))
    nodes = mesh.nodes()
    model = sf.Model(mesh, sf.Material(*STEEL))
    for n, a, v in stretched(nodes):
        model.prescribe_displacement(n, a, v)
    if pre == "jacobi":
        opts = sf.StudyOptions(pcg=sf.PcgOptions(tolerance=1e-12))
    else:
        prec = sf.Precision.DOUBLE if pre == "double" else sf.Precision.MIXED
        opts = sf.StudyOptions(pcg=sf.PcgOptions(tolerance=1e-12), preconditioner=sf.MultigridOptions(precision=prec))
    st = sf.StaticStudy.new(model, opts)
    assert st.solve().kind == sf.Outcome.CONVERGED
    sol = st.solution()
    d = sol.displacements
    assert np.all(d[nodes[:, 0] == 1.0, 0] == STRETCH)
    assert np.all(d[nodes[:, 0] == 0.0, 0] == 0.0)
    corner = int(np.flatnonzero(np.all(nodes == 1.0, axis=1))[0])
    assert abs(d[corner, 1] - (-STEEL[1] * STRETCH)) < 1e-6 * STRETCH
    expected = STEEL[0] * STRETCH
    stress = sol.point_stresses["stress"]
    assert np.all(np.abs(stress[:, 0] - expected) < 1e-5 * expected)
    assert np.all(np.abs(stress[:, 1:]) < 1e-5 * expected)


def test_prescribed_cantilever_matches_oracle(oracle):
    size, div, E, nu = (10.0, 1.0, 1.0), (12, 3, 3), 200000.0, 0.3
    mesh = sf.box_tet_mesh((0, 0, 0), size, div)
    nodes = mesh.nodes()
    fixed = np.flatnonzero(np.abs(nodes[:, 0]) < ON_PLANE)
    tip = np.flatnonzero(np.abs(nodes[:, 0] - size[0]) < ON_PLANE)
    prescribed = [(int(n), 2, -0.01) for n in tip] + [(int(tip[0]), 1, 0.002)]
    model = sf.Model(mesh, sf.Material(E, nu))
    model.fix_nodes(fixed)
    faces = mesh.boundary_face_array()
    top = np.all(np.abs(nodes[faces["nodes"][:, :3], 2] - size[2]) < ON_PLANE, axis=1)
    model.add_face_tractions(faces[top], (0.0, 1.0, 0.0))
    for n, a, v in prescribed:
        model.prescribe_displacement(n, a, v)
    st = sf.StaticStudy.new(model, sf.StudyOptions(pcg=sf.PcgOptions(tolerance=1e-12),
                                                   preconditioner=sf.MultigridOptions(coarse_dofs=100,
                                                                                      precision=sf.Precision.DOUBLE)))
    omesh = oracle.Mesh.box(size, div)
    ofaces = [(int(f["tet"]), int(f["face"]), [int(x) for x in f["nodes"]]) for f in faces[top]]
    ref = oracle.Study(omesh, oracle.uniform(E, nu), oracle.default_options(tolerance=1e-12, coarse_dofs=100,
                                                                           precision=oracle.DOUBLE),
                       fixed, ofaces, [[0.0, 1.0, 0.0]] * len(ofaces), prescribed=prescribed)
    rs, cols, vals = st.matrix()
    ors, ocols, ovals = ref.matrix()
    assert np.array_equal(cols, ocols) and np.array_equal(vals.view(np.uint64), ovals.view(np.uint64))
    assert np.array_equal(st.rhs().view(np.uint64), ref.rhs().view(np.uint64))
    assert st.solve().kind == sf.Outcome.CONVERGED
    ref.solve()
    d, dr = st.displacements(), ref.displacements()
    assert float(np.linalg.norm(d - dr) / np.linalg.norm(dr)) <= 1e-10
    for n, a, v in prescribed:
        assert d[n, a] == v
