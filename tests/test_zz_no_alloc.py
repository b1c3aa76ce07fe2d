"""sf_study_energy_products (allocates nothing, scratch in a static device array) against the
existing system product sf_study_system_multiply, on two calls in a row (needs a B200).

This file is named to be collected last, so it also runs after every other GPU test in the
same process, with the scratch already used by nothing else.
"""
import numpy as np
import pytest

import solidfem_b200 as sf
from tests.helpers import mg_options, product_model

pytestmark = pytest.mark.gpu

MAX_VECTORS = 8
# Rows are summed in the same order by both kernels; the energies are fixed-order sums of the same
# products, so only the reduction tree differs from numpy's dot.
Y_RTOL = 1e-13
ENERGY_RTOL = 1e-12


def make_study(sell):
    _, model = product_model((10.0, 1.0, 1.0), (12, 3, 3), 200000.0, 0.3)
    return sf.StaticStudy.new(model, mg_options(sf.Precision.DOUBLE, sell_min_rows=1 if sell else 0))


def energy_products(study, xs):
    import torch

    count, n = xs.shape
    x = torch.from_numpy(xs).to("cuda:0")
    y = torch.full((count, n), float("nan"), dtype=torch.float64, device="cuda:0")
    e = torch.full((count,), float("nan"), dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    study.energy_products(x.data_ptr(), y.data_ptr(), e.data_ptr(), count)
    torch.cuda.synchronize()
    return y.cpu().numpy(), e.cpu().numpy()


def check_against_system_multiply(study, xs, ys, es):
    for k, xk in enumerate(xs):
        yk = study.system_multiply(xk)
        assert np.linalg.norm(ys[k] - yk) <= Y_RTOL * np.linalg.norm(yk), k
        ek = float(np.dot(xk, yk))
        assert abs(es[k] - ek) <= ENERGY_RTOL * abs(ek), (k, es[k], ek)


@pytest.mark.parametrize("sell", [False, True])
def test_energy_products_match_system_multiply_twice(sell):
    study = make_study(sell)
    n = study.report()["free_dofs"]
    rng = np.random.default_rng(11)
    first = rng.standard_normal((3, n))
    second = rng.standard_normal((MAX_VECTORS, n))
    y1, e1 = energy_products(study, first)
    y2, e2 = energy_products(study, second)
    check_against_system_multiply(study, first, y1, e1)
    check_against_system_multiply(study, second, y2, e2)
    # the same inputs again give the same bits (the arrival tickets went back to zero)
    y3, e3 = energy_products(study, first)
    assert np.array_equal(y3.view(np.uint64), y1.view(np.uint64))
    assert np.array_equal(e3.view(np.uint64), e1.view(np.uint64))


def test_energy_products_refusals():
    import torch

    study = make_study(False)
    n = study.report()["free_dofs"]
    x = torch.zeros((MAX_VECTORS + 1, n), dtype=torch.float64, device="cuda:0")
    y = torch.zeros_like(x)
    e = torch.zeros(MAX_VECTORS + 1, dtype=torch.float64, device="cuda:0")
    with pytest.raises(sf.SolidfemError) as err:
        study.energy_products(x.data_ptr(), y.data_ptr(), e.data_ptr(), MAX_VECTORS + 1)
    assert err.value.status == sf.Status.INVALID_ARGUMENT
    assert "8 vectors" in str(err.value)
    host = np.zeros(n)
    with pytest.raises(sf.SolidfemError) as err:
        study.energy_products(host.ctypes.data, y.data_ptr(), e.data_ptr(), 1)
    assert err.value.status == sf.Status.INVALID_ARGUMENT
    with pytest.raises(sf.SolidfemError) as err:
        study.energy_products(x.data_ptr(), x.data_ptr(), e.data_ptr(), 1)
    assert err.value.status == sf.Status.INVALID_ARGUMENT
    study.energy_products(x.data_ptr(), y.data_ptr(), e.data_ptr(), 0)  # nothing to do


def test_energy_products_refuse_a_short_buffer_and_keep_the_current_device():
    """A range must lie inside one device allocation, as the driver reports it (cuMemGetAddressRange;
    the driver knows allocations, not a sub-allocator's pieces of them, and may round a request up).
    y placed so its two vectors end 8 bytes past the allocation is refused; placed to end exactly at
    the allocation's end it is accepted."""
    import torch
    from cuda.bindings import driver, runtime as rt

    study = make_study(False)
    n = study.report()["free_dofs"]
    x = torch.zeros((2, n), dtype=torch.float64, device="cuda:0")
    e = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    before = torch.cuda.current_device()
    err_code, buf = rt.cudaMalloc(4 * n * 8)
    assert err_code == rt.cudaError_t.cudaSuccess
    try:
        err_code, base, size = driver.cuMemGetAddressRange(int(buf))
        assert err_code == driver.CUresult.CUDA_SUCCESS
        end = int(base) + int(size)
        with pytest.raises(sf.SolidfemError) as err:
            study.energy_products(x.data_ptr(), end - 2 * n * 8 + 8, e.data_ptr(), 2)
        assert err.value.status == sf.Status.INVALID_ARGUMENT
        study.energy_products(x.data_ptr(), end - 2 * n * 8, e.data_ptr(), 2)
        torch.cuda.synchronize()
        assert torch.cuda.current_device() == before
    finally:
        rt.cudaFree(buf)
    with pytest.raises(sf.SolidfemError) as err:
        study.energy_products(x.data_ptr(), x[1].data_ptr(), e.data_ptr(), 2)  # x's second vector is y's first
    assert err.value.status == sf.Status.INVALID_ARGUMENT
