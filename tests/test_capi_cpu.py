"""CPU-only checks of the product boundary: the C-ABI library loads, exports every symbol that
include/solidfem_b200.h declares, and its host-side mesh input matches the oracle's to the bit
(the node numbering decides the aggregates). No device is needed for these."""
import os
import re

import numpy as np
import pytest

import solidfem_b200 as sf

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "solidfem_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(sf_\w+)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if not n.endswith("_fn")))


def test_library_exports_every_declared_symbol():
    lib = sf.library()
    names = header_functions()
    assert len(names) >= 40
    for name in names:
        assert hasattr(lib, name), name
        assert name in sf.SIGNATURES, name
    assert lib.sf_abi_version() == 3


def test_status_messages():
    lib = sf.library()
    assert lib.sf_status_message(0) == b"ok"
    assert b"positive definite" in lib.sf_status_message(int(sf.Status.PCG_NOT_POSITIVE_DEFINITE))


@pytest.mark.parametrize("size,div", [((10.0, 1.0, 1.0), (12, 3, 3)), ((20.0, 20.0, 1.0), (8, 8, 2)),
                                      ((100.0, 10.0, 10.0), (20, 4, 4))])
def test_box_mesh_matches_oracle(oracle, size, div):
    mine = sf.box_tet_mesh((0, 0, 0), size, div)
    ref = oracle.Mesh.box(size, div)
    assert mine.node_count() == ref.node_count and mine.tet_count() == ref.tet_count
    assert mine.vertex_count() == ref.vertex_count
    assert np.array_equal(mine.nodes().view(np.uint64), ref.nodes().view(np.uint64))
    assert np.array_equal(mine.tets(), ref.tets())
    faces = [f.key() for f in mine.boundary_faces()]
    assert faces == ref.faces()


def test_box_config_sizes():
    """Element, node and DOF counts of the benchmark configurations."""
    m = sf.box_tet_mesh((0, 0, 0), (100.0, 10.0, 10.0), (20, 4, 4))
    assert (m.tet_count(), m.node_count()) == (1920, 3321)
    m = sf.box_tet_mesh((0, 0, 0), (100.0, 100.0, 0.8), (60, 60, 2))
    assert (m.tet_count(), m.node_count()) == (43200, 73205)


def test_mesh_refusals():
    with pytest.raises(sf.SolidfemError) as e:
        sf.box_tet_mesh((0, 0, 0), (1.0, 1.0, 1.0), (0, 1, 1))
    assert e.value.status == sf.Status.MESH_INVALID_BOX
    with pytest.raises(sf.SolidfemError) as e:
        sf.Mesh.from_linear([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], [[0, 2, 1, 3]])
    assert e.value.status == sf.Status.MESH_DEGENERATE_TET
    with pytest.raises(sf.SolidfemError) as e:
        sf.Mesh.from_linear([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [5, 5, 5]], [[0, 1, 2, 3]])
    assert e.value.status == sf.Status.MESH_UNUSED_NODE


def test_linear_mesh_matches_oracle(oracle):
    rng = np.random.default_rng(0)
    box = oracle.Mesh.box((2.0, 1.0, 1.0), (2, 1, 1))
    corners = box.tets()[:, :4].astype(np.uint32)
    pos = box.nodes()[: box.vertex_count] + rng.uniform(-0.05, 0.05, size=(box.vertex_count, 3))
    mine = sf.Mesh.from_linear(pos, corners)
    ref = oracle.Mesh.linear(pos, corners)
    assert np.array_equal(mine.nodes().view(np.uint64), ref.nodes().view(np.uint64))
    assert np.array_equal(mine.tets(), ref.tets())
