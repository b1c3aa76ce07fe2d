"""Studies on two device ordinals in one process (needs two GPUs; skipped with fewer): kernels
whose launches need more than 48 KB of shared memory opt in per device, so a study on the second
device solves like one on the first, to the bit."""
import numpy as np
import pytest

import solidfem_b200 as sf
from tests.helpers import mg_options, product_model

pytestmark = pytest.mark.gpu


def device_count():
    import torch

    return torch.cuda.device_count()


@pytest.mark.skipif("device_count() < 2")
def test_two_devices_in_one_process_give_the_same_bits():
    answers = []
    for device in (0, 1):
        _, model = product_model((20.0, 20.0, 1.0), (8, 8, 2), 200000.0, 0.3)
        options = mg_options(sf.Precision.DOUBLE)
        options.device = device
        study = sf.StaticStudy.new(model, options)
        assert study.solve().kind == sf.Outcome.CONVERGED
        answers.append(study.displacements())
    assert np.array_equal(answers[0].view(np.uint64), answers[1].view(np.uint64))
