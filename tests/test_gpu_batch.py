"""Batched solves (sf_study_solve_batch) against the same studies solved alone (needs a B200).

A batch runs every kernel of a conjugate gradient step as one grid over all its studies, each
masked by its own status; each study's answer must be the one it gets alone.
"""
import numpy as np
import pytest

import solidfem_b200 as sf
from tests.helpers import mg_options, product_model

pytestmark = pytest.mark.gpu

# Same depth, different sizes, loads and materials.
CASES = [
    ((10.0, 1.0, 1.0), (12, 3, 3), 200000.0, 0.30, (0.0, 3.0, -7.0)),
    ((12.0, 1.5, 1.0), (14, 3, 3), 70000.0, 0.33, (1.0, 0.0, -2.0)),
    ((10.0, 1.0, 1.0), (12, 3, 3), 3000.0, 0.36, (0.0, -1.0, 4.0)),
    ((11.0, 1.2, 1.2), (13, 3, 3), 120000.0, 0.28, (0.5, 0.5, -5.0)),
]


def make(case, precision=sf.Precision.MIXED, batchable=True):
    size, div, E, nu, traction = case
    _, model = product_model(size, div, E, nu, traction=traction)
    return sf.StaticStudy.new(model, mg_options(precision, 1e-9, batchable=batchable))


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("precision", [sf.Precision.MIXED, sf.Precision.DOUBLE])
def test_batch_matches_solo(precision):
    solo = []
    for case in CASES:
        st = make(case, precision, batchable=False)
        out = st.solve()
        assert out.kind == sf.Outcome.CONVERGED
        solo.append((out.progress.iteration, st.displacements()))
    batch = [make(case, precision) for case in CASES]
    results = sf.solve_batch(batch)
    for (out, status), st, (its, d) in zip(results, batch, solo):
        assert status == sf.Status.OK
        assert out.kind == sf.Outcome.CONVERGED
        assert abs(out.progress.iteration - its) <= 1
        assert rel(st.displacements(), d) <= 1e-10


def test_batch_twice_gives_the_same_bits():
    batch = [make(case) for case in CASES]
    sf.solve_batch(batch)
    first = [st.displacements() for st in batch]
    sf.solve_batch(batch)
    for st, d in zip(batch, first):
        assert np.array_equal(st.displacements().view(np.uint64), d.view(np.uint64))


def test_batch_refuses_mixed_structure():
    small = make(CASES[0])
    size, div, E, nu, traction = CASES[0]
    _, model = product_model(size, div, E, nu, traction=traction)
    shallow = sf.StaticStudy.new(model, mg_options(sf.Precision.MIXED, 1e-9, coarse_dofs=4000, batchable=True))
    assert len(shallow.levels()) != len(small.levels())
    with pytest.raises(sf.SolidfemError) as err:
        sf.solve_batch([small, shallow])
    assert err.value.status == sf.Status.INVALID_ARGUMENT
