"""Regenerate the fixtures in this folder from the reference checkout.

    python tests/golden/make_golden.py /path/to/thirring-rhmc

Copies the reference's rational-approximation coefficient files (data read
by dwf3d_lib.F90:205-209 through remez_common_subroutines.F90:20-35) and the
12^3 checkpoint used by tests/broken_tests/test_load.F90, and records the
checkpoint's known answers decoded from the file itself.  The GPU box has no
reference checkout, so the tests read only these copies.
"""
import json
import os
import shutil
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def decode_con(path, k=12, kt=12):
    """Fortran unformatted sequential record: len, theta (k,k,kt,3) float32, seed float64, len."""
    raw = open(path, "rb").read()
    n = 3 * k * k * kt
    (l1,) = struct.unpack("<i", raw[:4])
    theta = np.frombuffer(raw[4:4 + 4 * n], "<f4").reshape((k, k, kt, 3), order="F")
    (seed,) = struct.unpack("<d", raw[4 + 4 * n:12 + 4 * n])
    (l2,) = struct.unpack("<i", raw[12 + 4 * n:16 + 4 * n])
    assert l1 == l2 == 4 * n + 8, (l1, l2)
    return theta, seed


def main(ref):
    for f in ("remez2", "remez4", "remez2g", "remez4g"):
        shutil.copy(os.path.join(ref, f), os.path.join(HERE, f))
    con = os.path.join(ref, "tests", "e2e_tests", "samples", "cons", "con_12x12x12")
    shutil.copy(con, os.path.join(HERE, "con_12x12x12"))
    theta, seed = decode_con(con)
    kat = {"sum": float(theta.astype(np.float64).sum()), "max": float(theta.max()),
           "min": float(theta.min()), "seed": seed,
           "reference_test": "tests/broken_tests/test_load.F90:28-31 (sum -185.5681, max 5.015248, "
                             "min -5.267587, seed 196829593468928)"}
    json.dump(kat, open(os.path.join(HERE, "con_12x12x12.json"), "w"), indent=1)
    print(json.dumps(kat, indent=1))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/thirring-rhmc")
    main(sys.argv[1])
