"""Face-connected bodies in the constraint check (constraints.rs with quadratic.rs:129-166), on
the host before any device work: two cubes sharing a face are one body; two cubes apart, or
touching along an edge only, are two, and the second, held by nothing (or by a line of nodes), is
refused as SF_BODY_NOT_HELD naming its first tet."""
import numpy as np
import pytest

import solidfem_b200 as sf

# A hex split into six tets around its main diagonal (corner 0 to corner 6).
HEX = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
SPLIT = [(0, 1, 2, 6), (0, 2, 3, 6), (0, 3, 7, 6), (0, 7, 4, 6), (0, 4, 5, 6), (0, 5, 1, 6)]


def cubes(offsets):
    """Unit cubes at the given offsets; coincident corners are merged."""
    index, positions, tets = {}, [], []
    for off in offsets:
        ids = []
        for c in HEX:
            p = tuple(float(c[a] + off[a]) for a in range(3))
            if p not in index:
                index[p] = len(positions)
                positions.append(p)
            ids.append(index[p])
        for t in SPLIT:
            v = [np.array(positions[ids[k]]) for k in t]
            vol = np.dot(np.cross(v[1] - v[0], v[2] - v[0]), v[3] - v[0])
            tet = [ids[k] for k in t]
            if vol < 0:
                tet[1], tet[2] = tet[2], tet[1]
            tets.append(tet)
    return np.array(positions), np.array(tets)


def build(offsets):
    pos, tets = cubes(offsets)
    mesh = sf.Mesh.from_linear(pos, tets)
    nodes = mesh.nodes()
    model = sf.Model(mesh, sf.Material(1000.0, 0.3))
    model.fix_nodes(np.flatnonzero(np.abs(nodes[:, 0]) < 1e-12))
    model.add_nodal_force(int(np.argmax(nodes[:, 0])), (0.0, 0.0, -1.0))
    with pytest.raises(sf.SolidfemError) as err:
        sf.StaticStudy.new(model, sf.StudyOptions())  # no device here: the build stops at the first refusal
    return err.value


def test_cubes_apart_are_two_bodies():
    e = build([(0, 0, 0), (3, 0, 0)])
    assert e.status == sf.Status.BODY_NOT_HELD
    assert e.detail["tet"] == 6  # the second body's first tet


def test_cubes_sharing_a_face_are_one_body():
    e = build([(0, 0, 0), (1, 0, 0)])
    assert e.status != sf.Status.BODY_NOT_HELD


def test_cubes_touching_along_an_edge_are_two_bodies():
    # held along the shared edge only: a line of nodes leaves the second cube free to turn
    e = build([(0, 0, 0), (1, 1, 0)])
    assert e.status == sf.Status.BODY_NOT_HELD
    assert e.detail["tet"] == 6


def test_many_tets_take_the_parallel_path():
    # 14^3 joined cubes (16,464 tets: the threaded bucket pass) and one cube apart
    block = [(i, j, k) for i in range(14) for j in range(14) for k in range(14)]
    e = build(block + [(20, 0, 0)])
    assert e.status == sf.Status.BODY_NOT_HELD
    assert e.detail["tet"] == 6 * len(block)
