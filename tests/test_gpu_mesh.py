"""Meshes generated on the device (needs a B200) against the host builders, which the oracle pins
(tests/test_capi_cpu.py): the same node coordinates to the bit, the same ten-node tets, the same
boundary faces in the same order, and the same refusals with the same payloads
(crates/solidfem-mesh/src/{box_mesh.rs:22-80, tet.rs:59-109, quadratic.rs:24-124},
demo/wasm/src/part.rs:135-189). A study built from a generated mesh takes its arrays on the device
and gives the same operator and answer as one built from the host mesh; its consistent traction
load is summed on the device (crates/solidfem-elastic/src/loads.rs:10-41) to the same bits."""
import numpy as np
import pytest

import solidfem_b200 as sf
from solidfem_b200 import workloads as W
from tests.helpers import mg_options

pytestmark = pytest.mark.gpu


def same_mesh(a: sf.Mesh, b: sf.Mesh):
    assert a.vertex_count() == b.vertex_count()
    assert np.array_equal(a.nodes().view(np.uint64), b.nodes().view(np.uint64))
    assert np.array_equal(a.tets(), b.tets())
    fa, fb = a.boundary_face_array(), b.boundary_face_array()
    assert len(fa) == len(fb) and np.array_equal(fa, fb)


@pytest.mark.parametrize("origin,size,div", [
    ((0.0, 0.0, 0.0), (10.0, 1.0, 1.0), (12, 3, 3)),
    ((-1.5, 0.25, 3.0), (7.3, 2.9, 1.1), (7, 5, 3)),
    ((0.0, 0.0, 0.0), (100.0, 100.0, 0.8), (60, 60, 2)),
    ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (1, 1, 1)),
])
def test_box_mesh_matches_the_host_builder(origin, size, div):
    dev = sf.box_tet_mesh(origin, size, div, device=0)
    assert dev.device() == 0
    host = sf.box_tet_mesh(origin, size, div)
    assert host.device() is None
    same_mesh(dev, host)


def graded_lines(length, cells, wall=None, wall_cells=2):
    """part.rs:57-86: a solid axis cut evenly, a tube axis with wall_cells cells across each wall
    and as many across the hollow."""
    if wall is None:
        return [length * i / cells for i in range(cells + 1)]
    inner, step = length - 2.0 * wall, wall / wall_cells
    lines = [step * i for i in range(wall_cells + 1)]
    lines += [wall + inner * i / wall_cells for i in range(1, wall_cells)]
    lines += [length - wall + step * i for i in range(wall_cells + 1)]
    return lines


@pytest.mark.parametrize("wall_cells", [0, 2])
def test_part_mesh_matches_its_host_restatement(wall_cells):
    x = graded_lines(40.0, 16)
    y = graded_lines(12.0, 0, wall=1.5, wall_cells=2) if wall_cells else graded_lines(12.0, 5)
    z = graded_lines(9.0, 0, wall=1.2, wall_cells=2) if wall_cells else graded_lines(9.0, 4)
    dev = sf.part_tet_mesh(x, y, z, wall_cells, device=0)
    host = W.part_mesh_host(x, y, z, wall_cells)
    same_mesh(dev, host)
    if wall_cells:
        nodes = dev.nodes()
        assert dev.tet_count() < 6 * 16 * 6 * 6  # the hollow core's cells are gone
        core = (nodes[:, 1] > 1.5) & (nodes[:, 1] < 10.5) & (nodes[:, 2] > 1.2) & (nodes[:, 2] < 7.8)
        assert not core.any()


def test_serving_parts_match_on_host_and_device():
    seen = set()
    for r in W.serving_stream():
        if r.kind in seen or r.target_dofs > 80_000:
            continue
        seen.add(r.kind)
        same_mesh(W.build_mesh(r, device=0), W.build_mesh(r))
    assert seen == set(W.KINDS)


def refusal(fn):
    try:
        fn()
    except sf.SolidfemError as e:
        return e.status, {k: e.detail.get(k) for k in ("tet", "node", "value")}
    return None


@pytest.mark.parametrize("case", ["out_of_range", "degenerate", "flat", "unused", "non_manifold", "non_finite"])
def test_generated_refusals_match_the_host(case):
    box = sf.box_tet_mesh((0.0, 0.0, 0.0), (3.0, 2.0, 1.0), (3, 2, 1))
    pos = box.nodes()[:box.vertex_count()].copy()
    tets = box.tets()[:, :4].astype(np.uint32).copy()
    if case == "out_of_range":
        tets[5, 2] = len(pos) + 7
    elif case == "degenerate":
        tets[4, [1, 2]] = tets[4, [2, 1]]
    elif case == "flat":
        pos = np.vstack([pos, [[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.5, 0.5, 1e-14]]])
        n = len(pos)
        tets = np.vstack([tets, [[n - 4, n - 3, n - 2, n - 1]]]).astype(np.uint32)
    elif case == "unused":
        pos = np.vstack([pos, [[9.0, 9.0, 9.0]]])
    elif case == "non_manifold":
        tets = np.vstack([tets, tets[3:4]]).astype(np.uint32)
    elif case == "non_finite":
        pos[6, 1] = np.nan
    host = refusal(lambda: sf.Mesh.from_linear(pos, tets))
    dev = refusal(lambda: sf.Mesh.from_linear(pos, tets, device=0))
    assert host is not None and dev is not None
    assert dev[0] == host[0]
    payload = {"out_of_range": ("tet", "node"), "degenerate": ("tet", "value"), "flat": ("tet", "value"),
               "unused": ("node",), "non_manifold": (), "non_finite": ("node",)}[case]
    for k in payload:
        assert np.float64(dev[1][k]).tobytes() == np.float64(host[1][k]).tobytes(), (k, dev, host)


def plate_model(mesh):
    nodes = mesh.nodes()
    model = sf.Model(mesh, sf.Material(2000.0, 0.35))
    model.fix_nodes(np.nonzero(np.abs(nodes[:, 0]) < 1e-9)[0])
    faces = mesh.boundary_face_array()
    top = np.all(np.abs(nodes[faces["nodes"][:, :3], 2] - 0.8) < 1e-9, axis=1)
    model.add_face_tractions(faces[top], (0.0, 0.0, -0.01))
    return model


def test_a_study_from_a_generated_mesh_is_the_same_study():
    size, div = (100.0, 100.0, 0.8), (40, 40, 2)
    host = sf.StaticStudy.new(plate_model(sf.box_tet_mesh((0, 0, 0), size, div)), mg_options(sf.Precision.MIXED))
    dev = sf.StaticStudy.new(plate_model(sf.box_tet_mesh((0, 0, 0), size, div, device=0)),
                             mg_options(sf.Precision.MIXED))
    # the pattern built on the device (incidence, sorted unique columns) is the host's
    hr, hc, hv = host.matrix()
    dr, dc, dv = dev.matrix()
    assert np.array_equal(hr, dr) and np.array_equal(hc, dc)
    assert np.array_equal(hv.view(np.uint64), dv.view(np.uint64))
    # neither the generated mesh's arrays nor the pattern and incidence crossed the host link
    node_bytes = 24 * dev.mesh.node_count() + 40 * dev.mesh.tet_count()
    pattern_bytes = 4 * (len(hc) // 9) + 40 * dev.mesh.tet_count()
    assert dev.device_timing()["h2d_bytes"] <= host.device_timing()["h2d_bytes"] - node_bytes - pattern_bytes
    oh, od = host.solve(), dev.solve()
    assert oh.progress.iteration == od.progress.iteration
    assert np.array_equal(host.displacements().view(np.uint64), dev.displacements().view(np.uint64))


def loaded_model(mesh):
    """Two traction sets sharing edge nodes, forces on nodes inside and outside the loaded faces."""
    nodes = mesh.nodes()
    model = sf.Model(mesh, sf.Material(200000.0, 0.3))
    model.fix_nodes(np.nonzero(np.abs(nodes[:, 0]) < 1e-9)[0])
    faces = mesh.boundary_face_array()
    corner = nodes[faces["nodes"][:, :3]]
    end = np.all(np.abs(corner[:, :, 0] - 10.0) < 1e-9, axis=1)
    top = np.all(np.abs(corner[:, :, 2] - 1.0) < 1e-9, axis=1)
    model.add_face_tractions(faces[end], (0.0, 3.0, -7.0))
    model.add_face_tractions(faces[top], (0.5, 0.0, -1.25))
    tip = np.nonzero(np.abs(nodes[:, 0] - 10.0) < 1e-9)[0]
    for node in list(tip[:3]) + [int(len(nodes) // 2)]:
        model.add_nodal_force(int(node), (1.0, -2.0, 0.75))
    return model


def test_generated_traction_load_matches_the_host_and_the_oracle(oracle):
    size, div = (10.0, 1.0, 1.0), (12, 3, 3)
    host = sf.StaticStudy.new(loaded_model(sf.box_tet_mesh((0, 0, 0), size, div)), mg_options(sf.Precision.DOUBLE))
    dev = sf.StaticStudy.new(loaded_model(sf.box_tet_mesh((0, 0, 0), size, div, device=0)),
                             mg_options(sf.Precision.DOUBLE))
    assert np.array_equal(host.rhs().view(np.uint64), dev.rhs().view(np.uint64))
    assert np.any(dev.rhs() != 0.0)
    # the oracle's build_load on the same model (traction faces and forces in the same order)
    om = oracle.Mesh.box(size, div)
    on = om.nodes()
    end, top = oracle.faces_on_plane(om, 0, 10.0, on), oracle.faces_on_plane(om, 2, 1.0, on)
    tip = np.nonzero(np.abs(on[:, 0] - 10.0) < 1e-9)[0]
    forces = [(int(n), (1.0, -2.0, 0.75)) for n in list(tip[:3]) + [int(len(on) // 2)]]
    ref = oracle.Study(om, oracle.uniform(200000.0, 0.3), oracle.default_options(precision=oracle.DOUBLE),
                       oracle.nodes_on_plane(on, 0, 0.0), end + top,
                       [[0.0, 3.0, -7.0]] * len(end) + [[0.5, 0.0, -1.25]] * len(top), forces=forces)
    assert np.array_equal(ref.rhs().view(np.uint64), dev.rhs().view(np.uint64))


@pytest.mark.parametrize("precision", [sf.Precision.DOUBLE, sf.Precision.MIXED])
def test_generated_part_and_prescribed_studies_match_the_host(precision):
    """A hollow part (the serving stream's tube) and a model with prescribed displacements: the
    studies from the generated meshes assemble the host's operator and give the host's answer."""
    x = [40.0 * i / 24 for i in range(25)]
    y = [12.0 * j / 8 for j in range(9)]
    meshes = (sf.part_tet_mesh(x, y, y, 2, device=0), W.part_mesh_host(x, y, y, 2))
    answers = []
    for mesh in meshes:
        nodes = mesh.nodes()
        model = sf.Model(mesh, sf.Material(70000.0, 0.33))
        model.fix_nodes(np.nonzero(np.abs(nodes[:, 0]) < 1e-9)[0])
        faces = mesh.boundary_face_array()
        end = np.all(np.abs(nodes[faces["nodes"][:, :3], 0] - 40.0) < 1e-9, axis=1)
        model.add_face_tractions(faces[end], (0.0, 0.0, -2.0))
        corner = int(np.nonzero(np.all(np.abs(nodes - [40.0, 0.0, 0.0]) < 1e-9, axis=1))[0][0])
        model.prescribe_displacement(corner, 1, 0.001)
        st = sf.StaticStudy.new(model, mg_options(precision))
        out = st.solve()
        answers.append((st.matrix(), st.rhs(), out.progress.iteration, st.displacements()))
    (dm, dr, di, dx), (hm, hr, hi, hx) = answers
    for a, b in zip(dm, hm):
        assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))
    assert np.array_equal(dr.view(np.uint64), hr.view(np.uint64))
    assert di == hi and np.array_equal(dx.view(np.uint64), hx.view(np.uint64))


def umbrella(k=30):
    """A vertex at the origin shared by 2k tetrahedra (a ring of k points, one apex above and one
    below): 10 x 2k candidate columns for its row, more than the device pattern build sorts in
    shared memory, so the study falls back to the host build."""
    ring = [(np.cos(2 * np.pi * i / k), np.sin(2 * np.pi * i / k), 0.0) for i in range(k)]
    pos = np.array([(0.0, 0.0, 0.0)] + ring + [(0.0, 0.0, 1.0), (0.0, 0.0, -1.0)])
    top, bottom = k + 1, k + 2
    tets = []
    for i in range(k):
        a, b = 1 + i, 1 + (i + 1) % k
        for t in ((0, a, b, top), (0, b, a, bottom)):
            p = pos[list(t)]
            if np.linalg.det(p[1:] - p[0]) < 0:
                t = (t[0], t[2], t[1], t[3])
            tets.append(t)
    return pos, np.array(tets, dtype=np.uint32)


def test_a_row_too_wide_for_the_device_pattern_takes_the_host_build():
    pos, tets = umbrella()
    matrices = []
    for device in (0, None):
        mesh = sf.Mesh.from_linear(pos, tets, device=device)
        nodes = mesh.nodes()
        model = sf.Model(mesh, sf.Material(1000.0, 0.3))
        model.fix_nodes(np.nonzero(nodes[:, 2] < -0.99)[0].tolist() + [1, 1 + len(pos) // 3])
        model.add_nodal_force(len(pos) - 2, (0.0, 0.0, 1.0))
        st = sf.StaticStudy.new(model, sf.StudyOptions(pcg=sf.PcgOptions(tolerance=1e-10)))
        st.solve()
        matrices.append((st.matrix(), st.displacements()))
    (dm, dx), (hm, hx) = matrices
    for a, b in zip(dm, hm):
        assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))
    assert np.array_equal(dx.view(np.uint64), hx.view(np.uint64))


def test_a_refusal_after_the_device_pattern_releases_it():
    """A generated mesh whose model has no load is refused after its pattern was built on the
    device; the refusal is the host's, and the device keeps working (repeated, nothing leaks)."""
    mesh = sf.box_tet_mesh((0, 0, 0), (10.0, 1.0, 1.0), (40, 4, 4), device=0)
    nodes = mesh.nodes()
    for _ in range(5):
        model = sf.Model(mesh, sf.Material(200000.0, 0.3))
        model.fix_nodes(np.nonzero(np.abs(nodes[:, 0]) < 1e-9)[0])
        with pytest.raises(sf.SolidfemError) as e:
            sf.StaticStudy.new(model, mg_options(sf.Precision.MIXED))
        assert e.value.status == sf.Status.NO_EFFECTIVE_LOAD
    model = plate_model(sf.box_tet_mesh((0, 0, 0), (100.0, 100.0, 0.8), (20, 20, 2), device=0))
    assert sf.StaticStudy.new(model, mg_options(sf.Precision.MIXED)).solve().kind == sf.Outcome.CONVERGED
