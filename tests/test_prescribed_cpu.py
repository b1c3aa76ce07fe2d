"""Prescribed-component refusals happen on the host, before any device work (CPU)."""
import numpy as np
import pytest

import solidfem_b200 as sf
from tests.test_oracle_prescribed import CUBE_POINTS, CUBE_TETS, STEEL


def cube_model():
    mesh = sf.Mesh.from_linear(np.array(CUBE_POINTS, dtype=np.float64), np.array(CUBE_TETS, dtype=np.uint32))
    return mesh, sf.Model(mesh, sf.Material(*STEEL))


def test_components_that_leave_a_rigid_motion_are_refused_by_name():
    mesh, model = cube_model()
    for i, p in enumerate(mesh.nodes()):
        if p[0] == 0.0:
            model.prescribe_displacement(i, 0, 0.0)
    with pytest.raises(sf.SolidfemError) as err:
        sf.StudyBuilder(model, sf.StudyOptions())
    assert err.value.status == sf.Status.DOFS_DO_NOT_HOLD
    assert err.value.detail["rank"] < 6


def test_bad_prescribed_components_are_refused():
    mesh, model = cube_model()
    for i, p in enumerate(mesh.nodes()):
        for a in range(3):
            model.prescribe_displacement(i, a, 0.0)
    model.prescribe_displacement(0, 3, 0.0)
    with pytest.raises(sf.SolidfemError) as err:
        sf.StudyBuilder(model, sf.StudyOptions())
    assert err.value.status == sf.Status.AXIS_OUT_OF_RANGE
