"""Device results against the oracle on the same seeded inputs (needs a B200).

Bit-exact: the device FP64 assembly (matrix and load), the host setup over it (aggregates and
every level's matrices and prolongators). Within tolerance: the device V-cycle against the
oracle's cycle in the same precision, and the PCG answer against the oracle's solve, following
the reference's own device-vs-CPU bounds (crates/solidfem-solve/tests/solver/gpu_solve_execution.rs).
"""
import numpy as np
import pytest

import solidfem_b200 as sf
from tests.helpers import mg_options, oracle_study, product_model

pytestmark = pytest.mark.gpu

CASES = {
    "cantilever": ((10.0, 1.0, 1.0), (12, 3, 3), 200000.0, 0.3),
    "plate": ((20.0, 20.0, 1.0), (8, 8, 2), 200000.0, 0.3),
}


def build(name, precision, tolerance=1e-9, sell=False):
    """The case on the device; `sell` puts every operator in the SELL-32 layout (by default only
    operators of at least 32768 block rows use it, which these small cases never reach)."""
    size, div, E, nu = CASES[name]
    mesh, model = product_model(size, div, E, nu)
    study = sf.StaticStudy.new(model, mg_options(precision, tolerance, sell_min_rows=1 if sell else 0))
    return mesh, study


def oracle_for(O, name, precision, tolerance=1e-9):
    size, div, E, nu = CASES[name]
    return oracle_study(O, size, div, E, nu, O.default_options(tolerance=tolerance, coarse_dofs=100,
                                                                precision=precision))


@pytest.mark.parametrize("name", list(CASES))
def test_assembly_and_load_are_bit_exact(oracle, name):
    _, study = build(name, sf.Precision.DOUBLE)
    ref = oracle_for(oracle, name, oracle.DOUBLE)
    rs, cols, vals = study.matrix()
    ors, ocols, ovals = ref.matrix()
    assert np.array_equal(rs, ors) and np.array_equal(cols, ocols)
    assert np.array_equal(vals.view(np.uint64), ovals.view(np.uint64))
    assert np.array_equal(study.rhs().view(np.uint64), ref.rhs().view(np.uint64))


@pytest.mark.parametrize("name", list(CASES))
def test_hierarchy_is_bit_exact(oracle, name):
    _, study = build(name, sf.Precision.DOUBLE)
    ref = oracle_for(oracle, name, oracle.DOUBLE)
    mine, theirs = study.levels(), ref.levels()
    assert len(mine) == len(theirs)
    for lv, (a, b) in enumerate(zip(mine, theirs)):
        assert a["rows"] == b["rows"], lv
        assert np.array_equal(a["starts"], b["starts"]) and np.array_equal(a["columns"], b["columns"]), lv
        assert np.array_equal(a["values"].view(np.uint64), b["values"].view(np.uint64)), lv
        assert a["lambda_max"] == b["lambda_max"], lv
        if "aggregates" in b:
            assert np.array_equal(a["aggregates"], b["aggregates"]), lv
            assert np.array_equal(a["p_columns"], b["p_columns"]), lv
            assert np.array_equal(a["p_values"].view(np.uint64), b["p_values"].view(np.uint64)), lv


@pytest.mark.parametrize("sell", [False, True])
@pytest.mark.parametrize("precision,tol", [(sf.Precision.DOUBLE, 1e-11), (sf.Precision.SINGLE_STORAGE, 1e-5),
                                           (sf.Precision.SINGLE, 1e-4)])
def test_device_cycle_matches_oracle_cycle(oracle, precision, tol, sell):
    """One V-cycle on the device against the oracle's cycle in the same precision."""
    opr = {sf.Precision.DOUBLE: oracle.DOUBLE, sf.Precision.SINGLE_STORAGE: oracle.SINGLE_STORAGE,
           sf.Precision.SINGLE: oracle.SINGLE}[precision]
    _, study = build("plate", precision, sell=sell)
    ref = oracle_for(oracle, "plate", opr)
    r = np.random.default_rng(7).standard_normal(ref.n)
    z, zr = study.precondition(r), ref.precondition(r)
    rel = np.linalg.norm(z - zr) / np.linalg.norm(zr)
    print(f"cycle {precision.name}: relative difference {rel:.3e}")
    assert rel <= tol


@pytest.mark.parametrize("sell", [False, True])
def test_system_multiply_matches_oracle(oracle, sell):
    _, study = build("cantilever", sf.Precision.DOUBLE, sell=sell)
    ref = oracle_for(oracle, "cantilever", oracle.DOUBLE)
    x = np.random.default_rng(3).standard_normal(ref.n)
    y, yr = study.system_multiply(x), ref.system_multiply(x)
    assert np.linalg.norm(y - yr) <= 1e-13 * np.linalg.norm(yr)


@pytest.mark.parametrize("sell", [False, True])
@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("precision", [sf.Precision.DOUBLE, sf.Precision.SINGLE_STORAGE, sf.Precision.SINGLE,
                                       sf.Precision.MIXED])
def test_solve_matches_oracle(oracle, name, precision, sell):
    mesh, study = build(name, precision, sell=sell)
    out = study.solve()
    assert out.kind == sf.Outcome.CONVERGED
    ref = oracle_for(oracle, name, oracle.DOUBLE)
    pr = ref.solve()
    d, dr = study.displacements(), ref.displacements()
    rep = study.report()
    print(f"{name} {precision.name}: iterations {out.progress.iteration} (oracle f64 {pr.iteration}), "
          f"residual {out.progress.relative_residual:.3e} floor {out.progress.at_rounding_floor}, "
          f"max diff / max {np.abs(d - dr).max() / np.abs(dr).max():.3e}")
    # The reference's device-solve cap: at most 2 cpu + 2 iterations (gpu_solve_execution.rs:145-160).
    assert out.progress.iteration <= 2 * pr.iteration + 2
    assert out.progress.relative_residual <= 1e-9 or out.progress.at_rounding_floor
    # Both stop at 1e-9 (or the floor): the reference's own 2e-3-of-largest bound between solves
    # (multigrid_precision.rs:110-125).
    assert np.abs(d - dr).max() <= 2e-3 * np.abs(dr).max()
    # The true residual of the device answer, measured with the oracle's FP64 product.
    x = d[ref.free_numbering() != 0xFFFFFFFF].reshape(-1)
    res = np.linalg.norm(ref.rhs() - ref.system_multiply(x)) / np.linalg.norm(ref.rhs())
    assert res <= 1e-9 or out.progress.at_rounding_floor
    assert rep["iterations"] == out.progress.iteration


def test_tight_double_solve_agrees_to_1e8(oracle):
    """At a 1e-12 residual (or the floor) both answers sit within 1e-8 relative L2 of each other."""
    _, study = build("cantilever", sf.Precision.DOUBLE, tolerance=1e-12)
    study.solve()
    ref = oracle_for(oracle, "cantilever", oracle.DOUBLE, tolerance=1e-12)
    ref.solve()
    d, dr = study.displacements(), ref.displacements()
    rel = np.linalg.norm(d - dr) / np.linalg.norm(dr)
    print(f"tight cantilever relative L2 {rel:.3e}")
    assert rel <= 1e-8


@pytest.mark.parametrize("sell", [False, True])
def test_sliced_solve_gives_identical_bits(sell):
    _, one = build("plate", sf.Precision.MIXED, sell=sell)
    one.solve()
    _, sliced = build("plate", sf.Precision.MIXED, sell=sell)
    while sliced.step(3).kind == sf.Outcome.RUNNING:
        pass
    a, b = one.displacements(), sliced.displacements()
    assert one.report()["iterations"] == sliced.report()["iterations"]
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_cancel_stays_cancelled():
    _, study = build("plate", sf.Precision.DOUBLE)
    calls = []
    out = study.step(10, cancel=lambda: calls.append(1) or len(calls) > 3)
    assert out.kind == sf.Outcome.CANCELLED
    assert out.progress.iteration == 3
    again = study.step(10)
    assert again.kind == sf.Outcome.CANCELLED and again.progress.iteration == 3


def test_jacobi_tension_bar_is_exact():
    """nu = 0 bar in tension with the default Jacobi preconditioner (tension.rs:13-57)."""
    length, force, E = 20.0, 1000.0, 2100.0
    mesh, model = product_model((length, 1.0, 1.0), (20, 2, 2), E, 0.0, traction=(force, 0.0, 0.0))
    study = sf.StaticStudy.new(model)
    assert study.solve().kind == sf.Outcome.CONVERGED
    nodes, d = mesh.nodes(), study.displacements()
    tip = np.abs(nodes[:, 0] - length) < 1e-9
    expected = force * length / E
    assert abs(d[tip, 0].mean() - expected) / expected < 1e-5


@pytest.mark.parametrize("name", list(CASES))
def test_fourteen_point_assembly_and_recovery_are_bit_exact(oracle, name):
    """The 14-point rule (quadrature.rs:53-161) through device assembly and recovery, to the bit
    against the oracle; on these straight-sided elements it also agrees with the 4-point rule to
    rounding (the integrand is quadratic: element/rigid_body.rs:129-139)."""
    size, div, E, nu = CASES[name]
    mesh, model = product_model(size, div, E, nu)
    model.set_quadrature(sf.Quadrature.FOURTEEN_POINT)
    study = sf.StaticStudy.new(model, mg_options(sf.Precision.DOUBLE))
    ref = oracle_study(oracle, size, div, E, nu, oracle.default_options(tolerance=1e-9, coarse_dofs=100,
                                                                        precision=oracle.DOUBLE, quadrature=1))
    _, _, vals = study.matrix()
    _, _, ovals = ref.matrix()
    assert np.array_equal(vals.view(np.uint64), ovals.view(np.uint64))
    _, four = product_model(size, div, E, nu)
    _, _, vals4 = sf.StaticStudy.new(four, mg_options(sf.Precision.DOUBLE)).matrix()
    assert np.abs(vals - vals4).max() < 1e-12 * np.abs(vals4).max()
    assert study.solve().kind == sf.Outcome.CONVERGED
    sol = study.solution()
    assert len(sol.point_stresses) == 14 * mesh.tet_count()
    s6, vm = ref.recover_with(sol.displacements)
    assert np.array_equal(sol.nodal_stress.view(np.uint64), s6.view(np.uint64))
    assert np.array_equal(sol.nodal_von_mises.view(np.uint64), vm.view(np.uint64))


def test_an_invalid_material_is_refused_at_the_first_element_and_point():
    """A material field that is not a stable solid in part of the body (nu = 0.5 past x = 6) is refused
    during device assembly by name, at the element and integration point the reference's serial
    assembly meets first (element.rs:83-94, ElementFault::InvalidMaterial)."""
    mesh, model = product_model((10.0, 1.0, 1.0), (12, 3, 3), 1.0, 0.0,
                                material=lambda p: sf.Material(200000.0, 0.5 if p[0] > 6.0 else 0.3))
    with pytest.raises(sf.SolidfemError) as err:
        sf.StaticStudy.new(model, mg_options(sf.Precision.DOUBLE))
    assert err.value.status == sf.Status.ELEMENT_INVALID_MATERIAL
    # the integration point positions, in (element, point) order, from a valid solve of the same mesh
    _, valid = product_model((10.0, 1.0, 1.0), (12, 3, 3), 200000.0, 0.3)
    study = sf.StaticStudy.new(valid, mg_options(sf.Precision.DOUBLE))
    assert study.solve().kind == sf.Outcome.CONVERGED
    pts = study.solution().point_stresses
    first = int(np.flatnonzero(pts["position"][:, 0] > 6.0)[0])
    assert (err.value.detail["tet"], err.value.detail["point"]) == (pts["tet"][first], pts["point"][first])
