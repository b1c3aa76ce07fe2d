"""The coarse tail: the last smoothed level and the coarse direct solve run as one thread-block-cluster
launch. On the thin plate (levels of 72,600 / 25,380 / 460 / 38 block rows) it takes level 2, cuts
the launches per iteration, and returns the bits of the per-phase launches it replaces: the same
iteration count and bitwise-equal displacements."""
import numpy as np
import pytest

import solidfem_b200 as sf
from tests.helpers import product_model

pytestmark = pytest.mark.gpu

PLATE = ((100.0, 100.0, 0.8), (60, 60, 2), 2000.0, 0.35)
LOAD = dict(load_axis=2, load_value=0.8, traction=(0.0, 0.0, -0.01))


def solve(precision, tail):
    _, model = product_model(*PLATE, **LOAD)
    options = sf.StudyOptions(pcg=sf.PcgOptions(tolerance=1e-8), coarse_tail=tail,
                              preconditioner=sf.MultigridOptions(precision=precision))
    study = sf.StaticStudy.new(model, options)
    return study, study.solve()


# f64 storage needs more shared memory than a 16-CTA cluster holds: no tail there, the same bits
@pytest.mark.parametrize("precision,fused_expected", [(sf.Precision.MIXED, True), (sf.Precision.SINGLE_STORAGE, True),
                                                      (sf.Precision.DOUBLE, False)])
def test_tail_returns_the_per_phase_bits(precision, fused_expected):
    fused, fo = solve(precision, True)
    plain, po = solve(precision, False)
    ft, pt = fused.device_timing(), plain.device_timing()
    print(f"{precision.name}: tail level {ft['coarse_tail_level']} on {ft['coarse_tail_cluster']} CTAs, "
          f"{ft['launches_per_iteration']} vs {pt['launches_per_iteration']} launches per iteration, "
          f"{fo.progress.iteration} iterations")
    assert pt["coarse_tail_cluster"] == 0 and pt["coarse_tail_level"] == -1
    if fused_expected:
        assert ft["coarse_tail_cluster"] in (8, 16) and ft["coarse_tail_level"] == 2
        assert ft["launches_per_iteration"] < pt["launches_per_iteration"]
    assert fo.kind == po.kind == sf.Outcome.CONVERGED
    assert fo.progress.iteration == po.progress.iteration
    assert np.array_equal(fused.displacements().view(np.uint64), plain.displacements().view(np.uint64))


def test_tail_preconditioner_matches_bitwise():
    """One standalone V-cycle on a seeded residual: the fused and per-phase cycles agree bit for bit."""
    fused, _ = solve(sf.Precision.MIXED, True)
    plain, _ = solve(sf.Precision.MIXED, False)
    r = np.random.default_rng(0).standard_normal(fused.rhs().shape[0])
    zf, zp = fused.precondition(r), plain.precondition(r)
    assert np.isfinite(zf).all()
    assert np.array_equal(zf.view(np.uint64), zp.view(np.uint64))
