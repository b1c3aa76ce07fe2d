"""The oracle against the reference's own golden values (CPU only).

Pins: the f64 multigrid fingerprints and the pinned iteration counts of
crates/solidfem/tests/validation/multigrid_precision.rs:134-250, and the closed-form tension bar of
crates/solidfem/tests/validation/tension.rs:13-57.
"""
import numpy as np
import pytest


def loaded(O, size, divisions, precision):
    """Steel clamped at x = 0, traction (0, 3, -7) on the x = L faces (multigrid_precision.rs:25-33)."""
    mesh = O.Mesh.box(size, divisions)
    nodes = mesh.nodes()
    fixed = O.nodes_on_plane(nodes, 0, 0.0)
    faces = O.faces_on_plane(mesh, 0, size[0], nodes)
    opts = O.default_options(tolerance=1e-9, coarse_dofs=100, precision=precision)
    study = O.Study(mesh, O.uniform(200000.0, 0.3), opts, fixed, faces, [[0.0, 3.0, -7.0]] * len(faces))
    progress = study.solve()
    assert progress.status == O.CONVERGED
    return study, progress


CASES = {
    "cantilever": ((10.0, 1.0, 1.0), (12, 3, 3)),
    "plate": ((20.0, 20.0, 1.0), (8, 8, 2)),
}


@pytest.mark.parametrize("name,expected", [("cantilever", (61, 4639424340864456019)),
                                           ("plate", (85, 5373319653865270473))])
def test_f64_cycle_fingerprint(oracle, name, expected):
    study, progress = loaded(oracle, *CASES[name], oracle.DOUBLE)
    assert (progress.iteration, study.fingerprint()) == expected
    # The same hash computed independently from the displacement array.
    assert oracle.fnv1a(study.displacements()) == expected[1]


@pytest.mark.parametrize("name,precision,iterations,floor", [
    ("cantilever", "SINGLE_STORAGE", 61, False), ("cantilever", "SINGLE", 65, False),
    ("plate", "SINGLE_STORAGE", 85, True), ("plate", "SINGLE", 90, True)])
def test_pinned_iteration_counts(oracle, name, precision, iterations, floor):
    double, dp = loaded(oracle, *CASES[name], oracle.DOUBLE)
    assert bool(dp.at_rounding_floor) == floor
    study, progress = loaded(oracle, *CASES[name], getattr(oracle, precision))
    assert progress.iteration == iterations
    assert progress.relative_residual <= 1e-9 or progress.at_rounding_floor
    a, b = double.displacements(), study.displacements()
    assert np.abs(a - b).max() <= 2e-3 * np.abs(a).max()
    assert study.stats()["memory_bytes"] < double.stats()["memory_bytes"]


def test_threads_do_not_change_bits(oracle):
    oracle.set_threads(1)
    one, _ = loaded(oracle, *CASES["plate"], oracle.SINGLE_STORAGE)
    oracle.set_threads(4)
    four, _ = loaded(oracle, *CASES["plate"], oracle.SINGLE_STORAGE)
    oracle.set_threads(1)
    assert one.fingerprint() == four.fingerprint()


def test_tension_bar_is_exact(oracle):
    """nu = 0 bar in tension, Jacobi PCG at 1e-9 (tension.rs:13-57)."""
    O = oracle
    length, force, E = 20.0, 1000.0, 2100.0
    mesh = O.Mesh.box((length, 1.0, 1.0), (20, 2, 2))
    nodes = mesh.nodes()
    faces = O.faces_on_plane(mesh, 0, length, nodes)
    study = O.Study(mesh, O.uniform(E, 0.0), O.default_options(preconditioner=O.JACOBI),
                    O.nodes_on_plane(nodes, 0, 0.0), faces, [[force, 0.0, 0.0]] * len(faces))
    assert study.solve().status == O.CONVERGED
    d = study.displacements()
    tip = O.nodes_on_plane(nodes, 0, length)
    elongation = d[tip, 0].mean()
    expected = force * length / E
    assert abs(elongation - expected) / expected < 1e-5
    s6, vm = study.recover()
    for p in study.point_stresses():
        assert abs(p.stress[0] - force) / force < 1e-5
        assert abs(p.von_mises - force) / force < 1e-5
    assert np.all(np.abs(vm - force) / force < 1e-5)
