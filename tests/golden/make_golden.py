"""Write ``oracle_golden.npz``: the CPU oracle's outputs on the seeded cases
of ``golden_cases.py`` (test infrastructure; run from the repository root):

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from golden_cases import CASES  # noqa: E402


def main():
    out = {}
    for name, fn in CASES.items():
        for key, arr in fn("oracle").items():
            out[f"{name}/{key}"] = np.ascontiguousarray(arr)
    path = os.path.join(HERE, "oracle_golden.npz")
    np.savez_compressed(path, **out)
    print(f"{path}: {len(out)} arrays, {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
