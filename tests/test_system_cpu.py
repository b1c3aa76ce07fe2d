"""Raw-system refusals (sf_system_create) that come before any device work, so they run without a
GPU: a malformed CSR matrix, the multigrid setup's named length and block-structure errors
(crates/solidfem-solve/tests/solver/multigrid.rs:42-103, multigrid/setup.rs:129-160,
block.rs:51-99) and Jacobi's non-positive diagonal (preconditioner.rs:49-79)."""
import numpy as np
import pytest

import solidfem_b200 as sf
from tests.system_cases import block_chain, csr, laplacian, modes_for, positions_for, unit_end_load


def mg():
    return sf.StudyOptions(preconditioner=sf.MultigridOptions())


def refused(status, *args, **kw):
    with pytest.raises(sf.SolidfemError) as err:
        sf.System(*args, **kw)
    assert err.value.status == status, err.value
    return err.value.detail


def test_a_near_null_space_of_the_wrong_length_is_refused_by_name():
    rs, cols, vals = block_chain(4)
    n = len(rs) - 1
    d = refused(sf.Status.MG_NEAR_NULL_LENGTH, rs, cols, vals, np.ones(n), mg(), near_null=modes_for(n - 3),
                positions=positions_for(4))
    assert (d["expected"], d["found"]) == (6 * n, 6 * (n - 3))


def test_positions_of_the_wrong_length_are_refused_by_name():
    rs, cols, vals = block_chain(4)
    n = len(rs) - 1
    d = refused(sf.Status.MG_POSITION_LENGTH, rs, cols, vals, np.ones(n), mg(), near_null=modes_for(n),
                positions=positions_for(3))
    assert (d["expected"], d["found"]) == (4, 3)


def test_a_matrix_without_three_by_three_blocks_is_refused_by_name():
    # a scalar chain of six unknowns: rows 0, 1, 2 do not share one pattern of whole blocks
    rs, cols, vals = laplacian(6)
    d = refused(sf.Status.MG_BLOCK_STRUCTURE, rs, cols, vals, np.ones(6), mg(), near_null=modes_for(6),
                positions=positions_for(2))
    assert d["row"] == 1
    rs, cols, vals = laplacian(7)
    d = refused(sf.Status.MG_BLOCK_STRUCTURE, rs, cols, vals, np.ones(7), mg(), near_null=modes_for(7),
                positions=positions_for(2))
    assert d["row"] == 7


def test_jacobi_refuses_a_diagonal_that_is_not_positive():
    rs, cols, vals = csr(3, {(0, 0): 2.0, (1, 1): -1.0, (2, 2): 2.0})
    d = refused(sf.Status.JACOBI_DIAGONAL, rs, cols, vals, np.ones(3))
    assert d["row"] == 1 and d["value"] == -1.0
    rs, cols, vals = csr(3, {(0, 0): 2.0, (2, 2): 2.0})  # row 1 has no diagonal entry
    d = refused(sf.Status.JACOBI_DIAGONAL, rs, cols, vals, np.ones(3))
    assert d["row"] == 1


def test_malformed_csr_is_refused():
    rs, cols, vals = laplacian(5)
    bad = cols.copy()
    bad[1], bad[2] = bad[2], bad[1]  # row 1's columns out of order
    refused(sf.Status.INVALID_ARGUMENT, rs, bad, vals, unit_end_load(5))
    bad = cols.copy()
    bad[-1] = 9  # a column past n
    refused(sf.Status.INVALID_ARGUMENT, rs, bad, vals, unit_end_load(5))
    with pytest.raises(ValueError):
        sf.System(rs, cols, vals, np.ones(4))
