"""Device stress recovery against the oracle (needs a B200).

The recovery of the same displacements must equal the oracle's to the bit (every step of
crates/solidfem-elastic/src/results.rs and patch.rs runs in the reference's order), including a
two-material part whose interface patches fall back to the worst incident element value; and
the closed-form tension bar reads its axial stress at every node (tension.rs:13-57).
"""
import numpy as np
import pytest

import solidfem_b200 as sf
from tests.helpers import mg_options, oracle_study, product_model

pytestmark = pytest.mark.gpu


def check_recovery_bits(oracle, study, ref):
    sol = study.solution()
    s6, vm = ref.recover_with(sol.displacements)
    assert np.array_equal(sol.nodal_stress.view(np.uint64), s6.view(np.uint64))
    assert np.array_equal(sol.nodal_von_mises.view(np.uint64), vm.view(np.uint64))
    pts = ref.point_stresses()
    got = sol.point_stresses
    assert len(got) == len(pts)
    ref_stress = np.array([list(p.stress) for p in pts])
    ref_vm = np.array([p.von_mises for p in pts])
    assert np.array_equal(got["stress"].view(np.uint64), ref_stress.view(np.uint64))
    assert np.array_equal(got["von_mises"].view(np.uint64), ref_vm.view(np.uint64))
    return sol


@pytest.mark.parametrize("size,div", [((10.0, 1.0, 1.0), (12, 3, 3)), ((20.0, 20.0, 1.0), (8, 8, 2))])
def test_recovery_is_bit_exact(oracle, size, div):
    _, model = product_model(size, div, 200000.0, 0.3)
    study = sf.StaticStudy.new(model, mg_options(sf.Precision.MIXED))
    assert study.solve().kind == sf.Outcome.CONVERGED
    ref = oracle_study(oracle, size, div, 200000.0, 0.3, oracle.default_options(tolerance=1e-9, coarse_dofs=100))
    check_recovery_bits(oracle, study, ref)


def test_two_material_recovery_is_bit_exact(oracle):
    """A shell/core block: patches that straddle the interface are left unfitted and read the
    worst incident element value (results.rs:43-46)."""
    size, div = (6.0, 6.0, 6.0), (6, 6, 6)
    lo, hi = (0.0, 0.0, 0.0), size
    mat = sf.ShellCore(sf.Material(2400.0, 0.36), sf.Material(800.0, 0.30), lo, hi, 2.0)
    _, model = product_model(size, div, 0, 0, clamp_axis=2, clamp_value=0.0, load_axis=2, load_value=size[2],
                             traction=(0.5, 0.0, 0.0), material=mat)
    study = sf.StaticStudy.new(model, mg_options(sf.Precision.DOUBLE))
    assert study.solve().kind == sf.Outcome.CONVERGED
    omat = oracle.shell_core((2400.0, 0.36), (800.0, 0.30), lo, hi, 2.0)
    ref = oracle_study(oracle, size, div, 0, 0, oracle.default_options(tolerance=1e-9, coarse_dofs=100),
                       clamp_axis=2, clamp_value=0.0, load_axis=2, load_value=size[2], traction=(0.5, 0.0, 0.0),
                       material=omat)
    _, _, vals = study.matrix()
    _, _, ovals = ref.matrix()
    assert np.array_equal(vals.view(np.uint64), ovals.view(np.uint64))
    check_recovery_bits(oracle, study, ref)


def test_tension_bar_nodal_von_mises_is_exact():
    length, force, E = 20.0, 1000.0, 2100.0
    _, model = product_model((length, 1.0, 1.0), (20, 2, 2), E, 0.0, traction=(force, 0.0, 0.0))
    study = sf.StaticStudy.new(model)
    assert study.solve().kind == sf.Outcome.CONVERGED
    sol = study.solution()
    assert np.all(np.abs(sol.point_stresses["stress"][:, 0] - force) / force < 1e-5)
    assert np.all(np.abs(sol.point_stresses["von_mises"] - force) / force < 1e-5)
    assert np.all(np.abs(sol.nodal_von_mises - force) / force < 1e-5)


def test_solution_refused_before_convergence():
    _, model = product_model((10.0, 1.0, 1.0), (12, 3, 3), 200000.0, 0.3)
    study = sf.StaticStudy.new(model, mg_options(sf.Precision.DOUBLE))
    study.step(2)
    with pytest.raises(sf.SolidfemError) as e:
        study.solution()
    assert e.value.status == sf.Status.NOT_FINISHED


def field_bits(f):
    return [np.ascontiguousarray(a).view(np.uint8) for a in
            (f.displacements, f.nodal_stress, f.nodal_von_mises, f.point_stresses)]


def assert_same_field(a, b):
    for x, y in zip(field_bits(a), field_bits(b)):
        assert np.array_equal(x, y)


def recover_in_slices(study, budget, cancel_at=None):
    rec = study.begin_recovery()
    calls = 0
    while True:
        calls += 1
        if cancel_at is not None and calls == cancel_at:
            with pytest.raises(sf.SolidfemError) as err:
                rec.continue_(budget, cancel=lambda: True)
            assert err.value.status == sf.Status.CANCELLED
            continue
        if rec.continue_(budget):
            return rec.finish()


@pytest.mark.parametrize("budget", [1, 97, 1000, 2**40])
def test_sliced_recovery_gives_the_bits_of_one_call(budget):
    """continue_recovery in any slices (results.rs:97-124: a recovery resumed in slices gives
    exactly the bits of one run), with a cancelled call in the middle that changes nothing."""
    _, model = product_model((10.0, 1.0, 1.0), (12, 3, 3), 200000.0, 0.3)
    study = sf.StaticStudy.new(model, mg_options(sf.Precision.MIXED))
    assert study.solve().kind == sf.Outcome.CONVERGED
    whole = study.solution()
    sliced = recover_in_slices(study, budget, cancel_at=2 if budget < 2**40 else None)
    assert_same_field(whole, sliced)


def test_a_preview_recovery_runs_before_convergence_and_matches_the_oracle(oracle):
    """begin_recovery on a solve still running recovers the estimate so far (a preview), bit-exact
    with the oracle's recovery of those displacements; solution() still refuses."""
    size, div = (20.0, 20.0, 1.0), (8, 8, 2)
    _, model = product_model(size, div, 200000.0, 0.3)
    study = sf.StaticStudy.new(model, mg_options(sf.Precision.DOUBLE))
    assert study.step(5).kind == sf.Outcome.RUNNING
    rec = study.begin_recovery()
    with pytest.raises(sf.SolidfemError) as err:
        rec.finish()
    assert err.value.status == sf.Status.NOT_FINISHED
    while not rec.continue_(500):
        pass
    field = rec.finish()
    assert np.array_equal(field.displacements.view(np.uint64), study.displacements().view(np.uint64))
    ref = oracle_study(oracle, size, div, 200000.0, 0.3, oracle.default_options(tolerance=1e-9, coarse_dofs=100))
    s6, vm = ref.recover_with(field.displacements)
    assert np.array_equal(field.nodal_stress.view(np.uint64), s6.view(np.uint64))
    assert np.array_equal(field.nodal_von_mises.view(np.uint64), vm.view(np.uint64))
    with pytest.raises(sf.SolidfemError) as err:
        study.solution()
    assert err.value.status == sf.Status.NOT_FINISHED


def test_solution_can_be_cancelled():
    _, model = product_model((10.0, 1.0, 1.0), (12, 3, 3), 200000.0, 0.3)
    study = sf.StaticStudy.new(model, mg_options(sf.Precision.DOUBLE))
    assert study.solve().kind == sf.Outcome.CONVERGED
    with pytest.raises(sf.SolidfemError) as err:
        study.solution(cancel=lambda: True)
    assert err.value.status == sf.Status.CANCELLED
    sol = study.solution()  # nothing was kept from the cancelled call
    assert np.all(np.isfinite(sol.nodal_von_mises))


def test_a_recovery_outliving_its_study_can_still_be_destroyed():
    """Destroying the study first (as a garbage collector may) leaves the recovery handle valid for
    sf_recovery_destroy only."""
    _, model = product_model((10.0, 1.0, 1.0), (12, 3, 3), 200000.0, 0.3)
    study = sf.StaticStudy.new(model, mg_options(sf.Precision.DOUBLE))
    assert study.solve().kind == sf.Outcome.CONVERGED
    rec = study.begin_recovery()
    lib = sf.library()
    lib.sf_study_destroy(study._h)  # the study goes first
    study._h = None
    lib.sf_recovery_destroy(rec._h)
    rec._h = None
