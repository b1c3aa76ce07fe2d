"""Model refusals by name before any device work (ModelError, crates/solidfem-elastic/src/error.rs:
23-119; the reference refuses a model that is not held or has no effective load before solving,
study.rs:419-474): non-finite loads, no effective load, no fixed node, nodes that do not exist and a
component prescribed on a fixed node. None needs a GPU: StudyBuilder::new checks them first."""
import math

import numpy as np
import pytest

import solidfem_b200 as sf
from tests.helpers import product_model

SIZE, DIV = (10.0, 1.0, 1.0), (6, 2, 2)


def model():
    return product_model(SIZE, DIV, 200000.0, 0.3, traction=(0.0, 0.0, -1.0))


def refused(m, status):
    with pytest.raises(sf.SolidfemError) as err:
        sf.StudyBuilder(m, sf.StudyOptions())
    assert err.value.status == status, err.value
    return err.value.detail


@pytest.mark.parametrize("bad", [math.nan, math.inf, -math.inf])
def test_a_non_finite_nodal_force_is_refused(bad):
    mesh, m = model()
    m.add_nodal_force(mesh.node_count() - 1, (0.0, bad, 0.0))
    refused(m, sf.Status.NON_FINITE_LOAD)


def test_a_non_finite_traction_is_refused():
    mesh = sf.box_tet_mesh((0, 0, 0), SIZE, DIV)
    nodes = mesh.nodes()
    m = sf.Model(mesh, sf.Material(200000.0, 0.3))
    m.fix_nodes(np.flatnonzero(nodes[:, 0] == 0.0))
    face = next(f for f in mesh.boundary_faces() if all(nodes[n][0] == SIZE[0] for n in list(f.nodes)[:3]))
    m.add_traction(face, (math.nan, 0.0, 0.0))
    refused(m, sf.Status.NON_FINITE_LOAD)


def test_a_non_finite_prescribed_value_is_refused():
    mesh, m = model()
    m.prescribe_displacement(mesh.node_count() - 1, 0, math.nan)
    refused(m, sf.Status.NON_FINITE_LOAD)


def test_no_effective_load_is_refused():
    mesh = sf.box_tet_mesh((0, 0, 0), SIZE, DIV)
    nodes = mesh.nodes()
    m = sf.Model(mesh, sf.Material(200000.0, 0.3))
    m.fix_nodes(np.flatnonzero(nodes[:, 0] == 0.0))
    refused(m, sf.Status.NO_EFFECTIVE_LOAD)
    m.add_nodal_force(5, (0.0, 0.0, 0.0))  # a zero load is no load
    refused(m, sf.Status.NO_EFFECTIVE_LOAD)


def test_no_fixed_node_is_refused():
    mesh = sf.box_tet_mesh((0, 0, 0), SIZE, DIV)
    m = sf.Model(mesh, sf.Material(200000.0, 0.3))
    m.add_nodal_force(5, (0.0, 0.0, -1.0))
    refused(m, sf.Status.NO_FIXED_NODES)


def test_nodes_that_do_not_exist_are_refused_by_number():
    mesh, m = model()
    n = mesh.node_count()
    m.fix_node(n + 7)
    assert refused(m, sf.Status.NODE_OUT_OF_RANGE)["node"] == n + 7
    mesh, m = model()
    m.add_nodal_force(n, (1.0, 0.0, 0.0))
    assert refused(m, sf.Status.NODE_OUT_OF_RANGE)["node"] == n


def test_a_component_prescribed_on_a_fixed_node_is_refused():
    mesh, m = model()
    fixed = m.fixed[0]
    m.prescribe_displacement(fixed, 2, 0.1)
    assert refused(m, sf.Status.PRESCRIBED_ON_FIXED_NODE)["node"] == fixed
