"""Every stage of every level of the device V-cycle against the oracle's (needs a B200), on the
device's own input to that stage, within twice the per-entry rounding bound that the reference's
device tests derive (crates/solidfem-solve/src/gpu/reference.rs:256-355 for products and the
smoother; tests/solver/gpu_cycle_execution.rs:253-267 for a product followed by an addition;
the stage-by-stage walk of tests/solver/gpu_hierarchy_execution.rs:434-557). Each stage runs the
launches the cycle itself makes, fused smoother starts included, in every layout (row groups,
SELL-32, split rows) and precision. The unit of rounding is the vector type's: f32 for the
Single cycle, f64 for Double and SingleStorage.
"""
import numpy as np
import pytest

import solidfem_b200 as sf
from tests.helpers import mg_options, oracle_study, product_model

pytestmark = pytest.mark.gpu

CASES = {
    "plate": ((20.0, 20.0, 1.0), (8, 8, 2), 200000.0, 0.3),
    "cantilever": ((10.0, 1.0, 1.0), (12, 3, 3), 200000.0, 0.3),
}
PRECISIONS = [sf.Precision.DOUBLE, sf.Precision.SINGLE_STORAGE, sf.Precision.SINGLE]


def within(name, found, expected, bound):
    assert found.shape == expected.shape, name
    diff = np.abs(found - expected)
    worst = int(np.argmax(diff - 2.0 * bound))
    assert np.all(diff <= 2.0 * bound), (
        f"{name}: entry {worst} is {found[worst]!r} on the device and {expected[worst]!r} in the oracle, "
        f"bound {2.0 * bound[worst]:.3e}")
    return int(np.count_nonzero(found == expected))


def vector(rng, n, single):
    v = rng.standard_normal(n) * np.exp(rng.uniform(-2.0, 2.0, n))
    return v.astype(np.float32).astype(np.float64) if single else v


@pytest.mark.parametrize("layout", ["groups", "sell"])
@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("name", list(CASES))
def test_every_stage_is_within_its_rounding_bound(oracle, name, precision, layout):
    size, div, E, nu = CASES[name]
    _, model = product_model(size, div, E, nu)
    study = sf.StaticStudy.new(model, mg_options(precision, sell_min_rows=1 if layout == "sell" else 0))
    opr = {sf.Precision.DOUBLE: oracle.DOUBLE, sf.Precision.SINGLE_STORAGE: oracle.SINGLE_STORAGE,
           sf.Precision.SINGLE: oracle.SINGLE}[precision]
    ref = oracle_study(oracle, size, div, E, nu, oracle.default_options(tolerance=1e-9, coarse_dofs=100,
                                                                        precision=opr))
    levels = study.levels()
    assert len(levels) >= 3
    single = precision == sf.Precision.SINGLE
    rng = np.random.default_rng(5)
    S = sf.Stage
    total = identical = 0
    for lv, info in enumerate(levels):
        n = info["rows"] * info["row_block"]
        coarse = lv + 1 < len(levels)
        smoothed = coarse or not info["has_factor"]
        tag = f"{name} {precision.name} {layout} level {lv}"
        b, x = vector(rng, n, single), vector(rng, n, single)
        checks = []
        if smoothed:
            for stage, ostage, args in ((S.SMOOTH, oracle.STAGE_SMOOTH, (b,)), (S.START, oracle.STAGE_START, (b,)),
                                        (S.SMOOTH_ADD, oracle.STAGE_SMOOTH_ADD, (b, x))):
                found = study.level_stage(lv, stage, *args)
                checks.append((f"{tag} {stage.name}", found, *ref.level_stage(lv, ostage, *args)))
        r = study.level_stage(lv, S.RESIDUAL, b, x)
        checks.append((f"{tag} RESIDUAL", r, *ref.level_stage(lv, oracle.STAGE_RESIDUAL, b, x)))
        if smoothed:
            r2, d2 = study.level_stage(lv, S.RESIDUAL_START, b, x)
            checks.append((f"{tag} RESIDUAL_START residual", r2, *ref.level_stage(lv, oracle.STAGE_RESIDUAL, b, x)))
            checks.append((f"{tag} RESIDUAL_START start", d2, *ref.level_stage(lv, oracle.STAGE_START, r2)))
        if coarse:
            cinfo = levels[lv + 1]
            cn = cinfo["rows"] * cinfo["row_block"]
            c = study.level_stage(lv, S.RESTRICT, r, out_len=cn)
            checks.append((f"{tag} RESTRICT", c, *ref.level_stage(lv, oracle.STAGE_RESTRICT, r, out_len=cn)))
            if lv + 2 < len(levels) or not cinfo["has_factor"]:
                c2, s2 = study.level_stage(lv, S.RESTRICT_START, r, out_len=cn)
                checks.append((f"{tag} RESTRICT_START restriction", c2,
                               *ref.level_stage(lv, oracle.STAGE_RESTRICT, r, out_len=cn)))
                checks.append((f"{tag} RESTRICT_START start", s2, *ref.level_stage(lv + 1, oracle.STAGE_START, c2)))
            e = vector(rng, cn, single)
            p = study.level_stage(lv, S.PROLONG, e, x, out_len=n)
            checks.append((f"{tag} PROLONG", p, *ref.level_stage(lv, oracle.STAGE_PROLONG, e, x, out_len=n)))
        for what, found, expected, bound in checks:
            identical += within(what, found, expected, bound)
            total += len(found)
    print(f"{name} {precision.name} {layout}: {identical} of {total} stage values identical to the oracle's")
    # the device repeats a stage to the bit
    again = study.level_stage(0, S.SMOOTH, vector(np.random.default_rng(5), levels[0]["rows"] * 3, single))
    first = study.level_stage(0, S.SMOOTH, vector(np.random.default_rng(5), levels[0]["rows"] * 3, single))
    assert np.array_equal(again.view(np.uint64), first.view(np.uint64))
