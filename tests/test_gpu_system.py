"""The reference's solver unit tests on the device, through sf_system_* (needs a B200): the
conjugate gradient on the 1-D Laplacian with its closed-form answer, slicing, cancel, the
indefinite refusal, the rounding floor, the iteration cap (crates/solidfem-solve/tests/solver/
pcg.rs:8-126, pcg.rs:266-273), and the multigrid setup on the block chain: a solve, a cancelled
setup and a diagonal block that is not positive definite (tests/solver/multigrid.rs,
multigrid/setup.rs:286-305). Every failure here is made on the host: a matrix, a tolerance, a cap
or a cancel callback. None faults or stalls the device."""
import numpy as np
import pytest

import solidfem_b200 as sf
from tests.system_cases import block_chain, indefinite, laplacian, modes_for, positions_for, unit_end_load

pytestmark = pytest.mark.gpu


def options(tolerance=1e-9, max_iterations=None, multigrid=False, sell_min_rows=0, **mg):
    pre = sf.MultigridOptions(**mg) if multigrid else sf.Jacobi()
    return sf.StudyOptions(pcg=sf.PcgOptions(tolerance=tolerance, max_iterations=max_iterations), preconditioner=pre,
                           sell_min_rows=sell_min_rows)


def laplacian_system(n, **kw):
    rs, cols, vals = laplacian(n)
    return sf.System(rs, cols, vals, unit_end_load(n), options(**kw))


def exact(n):
    return np.arange(1, n + 1) / (n + 1)


@pytest.mark.parametrize("n", [49, 50, 51])  # n mod 3 = 1, 2, 0: padded to whole 3x3 blocks or not
@pytest.mark.parametrize("sell", [False, True])
def test_it_solves_a_system_with_a_known_solution(n, sell):
    s = laplacian_system(n, sell_min_rows=1 if sell else 0)
    out = s.step(10_000)
    assert out.kind == sf.Outcome.CONVERGED
    assert np.abs(s.estimate() - exact(n)).max() < 1e-8
    assert s.progress() == out.progress


def test_many_small_steps_give_identical_bits_to_one_long_run():
    whole = laplacian_system(80)
    whole.step(100_000)
    sliced = laplacian_system(80)
    while True:
        out = sliced.step(3)
        if out.kind == sf.Outcome.CONVERGED:
            break
        assert out.kind == sf.Outcome.RUNNING and out.progress.iteration > 0
        assert sliced.estimate().shape == (80,)  # a preview of the estimate so far
    assert np.array_equal(whole.estimate().view(np.uint64), sliced.estimate().view(np.uint64))


def test_cancel_stops_the_solve_and_it_stays_stopped():
    s = laplacian_system(50)
    s.step(3)
    out = s.step(1000, cancel=lambda: True)
    assert out.kind == sf.Outcome.CANCELLED and out.progress.iteration == 3
    assert s.step(1000).kind == sf.Outcome.CANCELLED


def test_an_indefinite_matrix_returns_a_specific_error():
    rs, cols, vals = indefinite()
    s = sf.System(rs, cols, vals, np.array([1.0, -1.0]))
    with pytest.raises(sf.SolidfemError) as err:
        s.step(100)
    assert err.value.status == sf.Status.PCG_NOT_POSITIVE_DEFINITE
    assert err.value.detail["curvature"] <= 0.0
    with pytest.raises(sf.SolidfemError) as again:  # a failure is sticky (pcg.rs:173-178)
        s.step(100)
    assert again.value.status == sf.Status.PCG_NOT_POSITIVE_DEFINITE


def test_a_tolerance_below_rounding_stops_at_the_floor_and_says_so():
    s = laplacian_system(50, tolerance=1e-18)
    out = s.step(100_000)
    assert out.kind == sf.Outcome.CONVERGED
    assert out.progress.at_rounding_floor and out.progress.relative_residual > 1e-18
    assert np.abs(s.estimate() - exact(50)).max() < 1e-10


def test_the_iteration_cap_gives_not_converged():
    s = laplacian_system(50, max_iterations=5)
    with pytest.raises(sf.SolidfemError) as err:
        s.step(1000)
    assert err.value.status == sf.Status.PCG_NOT_CONVERGED
    assert err.value.detail["iteration"] == 5 and err.value.detail["relative_residual"] > 1e-9
    with pytest.raises(sf.SolidfemError):
        s.step(1000)


def test_a_zero_right_hand_side_is_converged_at_once():
    rs, cols, vals = laplacian(10)
    s = sf.System(rs, cols, vals, np.zeros(10))
    out = s.step(10)
    assert out.kind == sf.Outcome.CONVERGED and out.progress.iteration == 0
    assert np.array_equal(s.estimate(), np.zeros(10))


def chain_system(nodes, precision=sf.Precision.DOUBLE, cancel=None, first_block=None, **kw):
    rs, cols, vals = block_chain(nodes, first_block)
    n = 3 * nodes
    rhs = np.sin(np.arange(n) * 0.37)
    s = sf.System(rs, cols, vals, rhs, options(multigrid=True, precision=precision, **kw),
                  near_null=modes_for(n), positions=positions_for(nodes), cancel=cancel)
    return s, (rs, cols, vals), rhs


@pytest.mark.parametrize("precision", list(sf.Precision))
def test_multigrid_solves_the_block_chain(precision):
    s, (rs, cols, vals), rhs = chain_system(3000, precision, tolerance=1e-10, coarse_dofs=300)
    assert s.level_count() >= 2
    out = s.solve()
    assert out.kind == sf.Outcome.CONVERGED
    x = s.estimate()
    n = len(rhs)
    ax = np.zeros(n)
    for r in range(n):
        lo, hi = int(rs[r]), int(rs[r + 1])
        ax[r] = np.dot(vals[lo:hi], x[cols[lo:hi]])
    assert np.linalg.norm(rhs - ax) <= 1e-10 * np.linalg.norm(rhs) * 1.0001 or out.progress.at_rounding_floor
    jac = sf.System(rs, cols, vals, rhs, options(tolerance=1e-12))
    jac.solve()
    assert np.abs(x - jac.estimate()).max() <= 1e-8 * np.abs(jac.estimate()).max()


def test_a_cancelled_setup_reports_cancelled():
    polls = []
    with pytest.raises(sf.SolidfemError) as err:
        chain_system(4000, cancel=lambda: polls.append(1) or len(polls) > 10)
    assert err.value.status == sf.Status.CANCELLED
    assert len(polls) >= 11


def test_a_diagonal_block_that_is_not_positive_definite_is_refused_by_name():
    # positive diagonal entries, eigenvalues 4, 4 and -2 in the first node's block
    bad = [[1.0, 3.0, 0.0], [3.0, 1.0, 0.0], [0.0, 0.0, 4.0]]
    with pytest.raises(sf.SolidfemError) as err:
        chain_system(40, first_block=bad)
    assert err.value.status == sf.Status.MG_NOT_POSITIVE_DEFINITE
    assert err.value.detail["level"] == 0 and err.value.detail["block"] == 0
