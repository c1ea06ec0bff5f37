"""Write tests/golden/ref_pin.npz: one-iteration cases whose expected values
come from TCLB's own model code (oracle/_ref, built from the reference tree by
oracle/make_ref.py). The cases are defined in tests/golden_cases.py.

    python tests/golden/make_golden.py        (needs the TCLB source tree)
"""
from __future__ import annotations

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.dirname(HERE)):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

import golden_cases  # noqa: E402


def main():
    out = golden_cases.generate()
    np.savez_compressed(golden_cases.FIXTURE, **out)
    print(golden_cases.FIXTURE, os.path.getsize(golden_cases.FIXTURE), "bytes")


if __name__ == "__main__":
    main()
