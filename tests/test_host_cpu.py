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


# ---- checkpoints (dwf3d_lib.F90:618-767); host code of the library, no GPU
def test_read_con_kat():
    # tests/broken_tests/test_load.F90:28-31 on the 12^3 sample configuration
    import json
    theta, seed, fmt = thirring.read_con(os.path.join(GOLD, "con_12x12x12"), 12, 12, 12)
    kat = json.load(open(os.path.join(GOLD, "con_12x12x12.json")))
    assert fmt == thirring.CON_SERIAL
    assert seed == 196829593468928.0 == kat["seed"]
    assert abs(theta.astype(np.float64).sum() - (-185.5681)) < 1e-3 * 185.5681
    assert abs(float(theta.max()) - 5.015248) < 1e-6 and abs(float(theta.min()) - (-5.267587)) < 1e-6


def test_con_round_trips(tmp_path):
    src = os.path.join(GOLD, "con_12x12x12")
    theta, seed, _ = thirring.read_con(src, 12, 12, 12)
    a = str(tmp_path / "con_serial")
    thirring.write_con(a, theta, seed, thirring.CON_SERIAL)
    assert open(a, "rb").read() == open(src, "rb").read()  # byte-identical to the reference's file
    b = str(tmp_path / "con_mpi")
    thirring.write_con(b, theta, seed, thirring.CON_MPIIO)
    raw = open(b, "rb").read()
    assert len(raw) == 4 * theta.size + 16
    assert raw[:4 * theta.size] == theta.tobytes(order="F")  # theta at offset 0
    t2, s2, fmt = thirring.read_con(b, 12, 12, 12)
    assert fmt == thirring.CON_MPIIO and s2 == seed and np.array_equal(t2, theta)
    with pytest.raises(thirring.ThirringError):
        thirring.read_con(src, 8, 8, 8)  # wrong lattice size


def test_seed_file_round_trip(tmp_path):
    p = str(tmp_path / "random_seed")
    for v in (4139764973254.0, 196829593468928.0, 1.0):
        thirring.saveseed(p, v)
        assert thirring.readseed(p) == v
    open(p, "w").write("   4139764973254.0000     \n")  # gfortran list-directed form
    assert thirring.readseed(p) == 4139764973254.0
