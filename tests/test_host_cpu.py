"""Host-side logic on CPU: the rational-approximation files the RHMC layer
feeds to thr_set_remez (read_remez_file, remez_common_subroutines.F90:20-35;
read at dwf3d_lib.F90:205-209)."""
import os

import numpy as np
import pytest

import oracle as O
import thirring

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILES = [("remez2", 25, 0.5, 1e-12), ("remez4", 25, 0.25, 1e-12),
         ("remez2g", 12, 0.5, 1e-6), ("remez4g", 12, 0.25, 1e-6)]


@pytest.mark.parametrize("name,n,power,tol", FILES)
def test_reader_matches_oracle(name, n, power, tol):
    path = os.path.join(GOLD, name)
    got = thirring.read_remez_file(path, n)
    ref = O.read_remez(path, n)
    for g, r in zip(got, ref):
        assert g.shape == r.shape
        assert np.array_equal(g, r)


@pytest.mark.parametrize("name,n,power,tol", FILES)
def test_sets_approximate_their_powers(name, n, power, tol):
    # set A ~ x^power and set B ~ x^-power over the spectral window the runs use
    a, ad, b, bd = thirring.read_remez_file(os.path.join(GOLD, name), n)
    x = np.logspace(-4.0, 1.5, 200)
    ra = a[0] + (a[1:, None] / (x[None, :] + ad[:, None])).sum(0)
    rb = b[0] + (b[1:, None] / (x[None, :] + bd[:, None])).sum(0)
    assert np.max(np.abs(ra / x ** power - 1)) < tol
    assert np.max(np.abs(rb * x ** power - 1)) < tol
    assert np.all(ad > 0) and np.all(bd > 0)


def test_remez_set_keys():
    rat = thirring.remez_set(os.path.join(GOLD, "remez2"), os.path.join(GOLD, "remez4"), 25)
    assert sorted(rat) == sorted(["anum2", "aden2", "bnum2", "bden2", "anum4", "aden4", "bnum4", "bden4"])
    assert all(len(rat[k]) == 26 for k in ("anum2", "bnum2", "anum4", "bnum4"))
    assert all(len(rat[k]) == 25 for k in ("aden2", "bden2", "aden4", "bden4"))
