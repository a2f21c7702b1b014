"""The CUDA path against the committed golden fixtures
(``tests/golden/oracle_golden.npz``, the CPU oracle's outputs on seeded
cases): bit for bit, including the Krylov iteration counts of the coupled
steps, without running the oracle."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, HERE)

from golden_cases import CASES  # noqa: E402

pytestmark = pytest.mark.gpu
GOLDEN = np.load(os.path.join(HERE, "oracle_golden.npz"))


@pytest.mark.parametrize("name", list(CASES))
def test_cuda_path_reproduces_golden(gpu, name):
    got = CASES[name]("gpu")
    keys = sorted(k.split("/", 1)[1] for k in GOLDEN.files if k.startswith(name + "/"))
    assert sorted(got) == keys
    for k in keys:
        np.testing.assert_array_equal(np.ascontiguousarray(got[k]), GOLDEN[f"{name}/{k}"], err_msg=f"{name}/{k}")
