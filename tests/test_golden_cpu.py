"""The CPU oracle against its committed golden fixtures
(``tests/golden/oracle_golden.npz``, written by ``tests/golden/make_golden.py``):
every array of every seeded case is reproduced bit for bit, so a change to
the oracle that alters its arithmetic is caught here, and the GPU parity
tests that read the same fixtures keep meaning what they meant."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, HERE)

from golden_cases import CASES  # noqa: E402

GOLDEN = np.load(os.path.join(HERE, "oracle_golden.npz"))


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_reproduces_golden(oracle_mod, name):
    got = CASES[name]("oracle")
    keys = sorted(k.split("/", 1)[1] for k in GOLDEN.files if k.startswith(name + "/"))
    assert sorted(got) == keys
    for k in keys:
        np.testing.assert_array_equal(np.ascontiguousarray(got[k]), GOLDEN[f"{name}/{k}"], err_msg=f"{name}/{k}")
