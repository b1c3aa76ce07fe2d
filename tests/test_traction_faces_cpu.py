"""Traction faces must be faces of the mesh boundary (study.rs:696-735, FaceNotOnBoundary), checked
on the host before any device work: the boundary's own faces pass; an interior face, a face whose
nodes are out of order, or a tet index past the mesh are refused."""
import numpy as np
import pytest

import solidfem_b200 as sf

# the six nodes of face f of a Tet10 in boundary-face order (corners, then midsides)
FACE_NODES = [(1, 2, 3, 5, 9, 8), (0, 3, 2, 7, 9, 6), (0, 1, 3, 4, 8, 7), (0, 2, 1, 6, 5, 4)]


def status_of(mesh, faces):
    nodes = mesh.nodes()
    model = sf.Model(mesh, sf.Material(1000.0, 0.3))
    model.fix_nodes(np.flatnonzero(np.abs(nodes[:, 0]) < 1e-12))
    model.add_face_tractions(faces, (0.0, 0.0, -1.0))
    with pytest.raises(sf.SolidfemError) as err:
        sf.StaticStudy.new(model, sf.StudyOptions())  # no device here: the build stops at the first refusal
    return err.value.status


@pytest.fixture(scope="module")
def mesh():
    return sf.box_tet_mesh((0.0, 0.0, 0.0), (2.0, 2.0, 2.0), (2, 2, 2))


def face_record(tets, t, f):
    rec = np.zeros(1, dtype=sf.FACE_DTYPE)
    rec["tet"], rec["face"] = t, f
    rec["nodes"][0] = [tets[t][k] for k in FACE_NODES[f]]
    return rec


def test_boundary_faces_pass(mesh):
    assert status_of(mesh, mesh.boundary_face_array()) != sf.Status.FACE_NOT_ON_BOUNDARY


def test_interior_face_refused(mesh):
    tets = mesh.tets()
    boundary = {(int(r["tet"]), int(r["face"])) for r in mesh.boundary_face_array()}
    t, f = next((t, f) for t in range(len(tets)) for f in range(4) if (t, f) not in boundary)
    assert status_of(mesh, face_record(tets, t, f)) == sf.Status.FACE_NOT_ON_BOUNDARY


def test_reordered_nodes_refused(mesh):
    faces = mesh.boundary_face_array()[:1].copy()
    faces["nodes"][0][[0, 1]] = faces["nodes"][0][[1, 0]]
    assert status_of(mesh, faces) == sf.Status.FACE_NOT_ON_BOUNDARY


def test_tet_past_the_mesh_refused(mesh):
    faces = mesh.boundary_face_array()[:1].copy()
    faces["tet"] = len(mesh.tets()) + 5
    assert status_of(mesh, faces) == sf.Status.FACE_NOT_ON_BOUNDARY
