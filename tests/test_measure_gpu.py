"""Device psibarpsi measurement (thr_measure) vs the oracle's restatement of
measure_module.F90:142-670, on the same links and random-number streams."""
import numpy as np
import pytest

import oracle as O
import thirring
from helpers import rand_links


def _run(dims, kernel_gen, kernel_meas, imass, res, am, u=None, seed=4139764973254.0, knoise=10, precision=0):
    L = O.lat(*dims, kernel=kernel_gen)
    if u is None:
        u = O.starting_state(L)["u"]
    g = O.RNG(L, True).init(seed)
    ref = O.measure(L, g, u, res, am, imass, kernel_meas=kernel_meas, knoise=knoise)
    with thirring.Lattice(*dims, kernel=kernel_gen) as G:
        G.set_links(u)
        G.init_random(seed)
        got = G.measure(res, am, imass, kernel_meas=kernel_meas, knoise=knoise, precision=precision)
    return ref, got


def _parts(ref):
    return np.array([[p1.real, p1.imag, p2.real, p2.imag] for p1, p2 in ref["parts"]])


@pytest.mark.gpu
def test_measure_shamir_fixture():
    # tests/test_measure_shamir.F90 set-up: every solve takes 5 iterations
    ref, got = _run((12, 12, 12, 24), 0, 0, 3, 0.1, 0.05)
    assert list(got["itercg"]) == ref["itercg"]
    assert got["aviter"] == ref["aviter"] == 5.0
    np.testing.assert_allclose(got["parts"], _parts(ref), rtol=1e-9, atol=1e-12)
    assert abs(got["psibarpsi"] - ref["psibarpsi"]) <= 1e-6 * abs(ref["psibarpsi"])
    assert abs(got["susclsing"] - ref["susclsing"]) <= 1e-5 * abs(ref["susclsing"])


@pytest.mark.gpu
@pytest.mark.parametrize("imass", [1, 3, 5])
def test_measure_shamir_converged(imass):
    # tight residual on random links: iteration counts within rounding, and the two
    # solutions (both meeting the stopping rule) agree to far below the estimator's noise
    dims = (6, 6, 8, 8)
    L = O.lat(*dims)
    u = rand_links(L, np.random.default_rng(40 + imass), beta=2.0)
    ref, got = _run(dims, 0, 0, imass, 1e-8, 0.1, u=u, seed=1234567.0, knoise=4)
    assert np.all(np.abs(np.array(got["itercg"]) - np.array(ref["itercg"])) <= 2)
    np.testing.assert_allclose(got["parts"], _parts(ref), rtol=1e-6, atol=1e-9)


@pytest.mark.gpu
def test_measure_wilson_on_shamir_generation():
    # MEASURE_WILSON with the Shamir generation kernel (the reference tests' build)
    ref, got = _run((12, 12, 12, 24), 0, 1, 3, 0.1, 0.05, knoise=4)
    assert list(got["itercg"]) == ref["itercg"]
    np.testing.assert_allclose(got["parts"], _parts(ref), rtol=1e-8, atol=1e-11)
    assert abs(got["psibarpsi"] - ref["psibarpsi"]) <= 1e-6 * abs(ref["psibarpsi"])


@pytest.mark.gpu
@pytest.mark.parametrize("imass", [1, 3])
def test_measure_wilson_wilson(imass):
    dims = (6, 6, 8, 8)
    L = O.lat(*dims, kernel=1)
    u = rand_links(L, np.random.default_rng(50 + imass), beta=2.0)
    ref, got = _run(dims, 1, 1, imass, 1e-8, 0.1, u=u, seed=987654321.0, knoise=3)
    assert np.all(np.abs(np.array(got["itercg"]) - np.array(ref["itercg"])) <= 2)
    np.testing.assert_allclose(got["parts"], _parts(ref), rtol=1e-6, atol=1e-9)


@pytest.mark.gpu
def test_measure_mixed_precision():
    # FP32 inner solves with FP64 defect correction: same estimate to the solver tolerance
    dims = (6, 6, 8, 8)
    L = O.lat(*dims)
    u = rand_links(L, np.random.default_rng(7), beta=2.0)
    ref, got = _run(dims, 0, 0, 3, 1e-8, 0.1, u=u, seed=1234567.0, knoise=3, precision=2)
    np.testing.assert_allclose(got["parts"], _parts(ref), rtol=1e-5, atol=1e-8)


@pytest.mark.gpu
def test_measure_rejects():
    with thirring.Lattice(4, 4, 4, 8) as G:
        G.set_links(O.starting_state(O.lat(4, 4, 4, 8))["u"])
        with pytest.raises(thirring.ThirringError):
            G.measure(0.1, 0.05, 3)  # no init_random yet
        G.init_random(1.0)
        with pytest.raises(thirring.ThirringError):
            G.measure(0.1, 0.05, 5, kernel_meas=1)  # measure_wilson has no imass 5 branch


@pytest.mark.gpu
def test_meson_fixture_kat():
    # tests/test_meson.F90: itercg == 3, aviter (3, 6, 6), and the correlators of the oracle
    dims = (12, 12, 12, 24)
    L = O.lat(*dims)
    u = O.starting_state(L)["u"]
    g = O.RNG(L, True).init(4139764973254.0)
    with thirring.Lattice(*dims) as G:
        G.set_links(u)
        G.init_random(4139764973254.0)
        for imass, aviter in ((1, 3.0), (3, 6.0), (5, 6.0)):
            ref = O.meson(L, g, u, 0.1, 0.05, imass)
            got = G.meson(0.1, 0.05, imass)
            assert got["itercg"] == 3 and got["aviter"] == aviter
            for k in ("cpm", "cmm", "cpmn", "cmmn"):
                np.testing.assert_allclose(got[k], ref[k], rtol=1e-9, atol=1e-14)
            assert abs(got["chim"] - ref["chim"]) <= 1e-9 * abs(ref["chim"])


@pytest.mark.gpu
@pytest.mark.parametrize("kernel,imass", [(0, 1), (0, 3), (0, 5), (1, 3)])
def test_meson_and_fermion_converged(kernel, imass):
    dims = (6, 6, 8, 8)
    L = O.lat(*dims, kernel=kernel)
    u = rand_links(L, np.random.default_rng(60 + imass), beta=2.0)
    g = O.RNG(L, True).init(24680.0)
    with thirring.Lattice(*dims, kernel=kernel) as G:
        G.set_links(u)
        G.init_random(24680.0)
        ref = O.meson(L, g, u, 1e-8, 0.1, imass, nsource=3)
        got = G.meson(1e-8, 0.1, imass, nsource=3)
        # both solutions meet congrad's absolute rule |r|^2 < 4 V Ls res^2; point and wall
        # sources have |xi| ~ 1, so they agree to ~1e-6 relative of the largest entry
        assert abs(got["itercg"] - ref["itercg"]) <= 2
        for k in ("cpm", "cmm", "cpmn", "cmmn"):
            np.testing.assert_allclose(got[k], ref[k], rtol=1e-5, atol=1e-6 * np.max(np.abs(ref[k])))
        ref = O.fermion(L, g, u, 1e-8, 0.1, imass, nsource=3)
        got = G.fermion(1e-8, 0.1, imass, nsource=3)
        for k in ("cferm1", "cferm2"):
            np.testing.assert_allclose(got[k], ref[k], rtol=1e-5, atol=1e-6 * np.max(np.abs(ref[k])))


def _measure_bits():
    """One Wilson-kernel measurement (the set-up of test_measure_wilson_wilson[1]) as exact bits."""
    dims = (6, 6, 8, 8)
    L = O.lat(*dims, kernel=1)
    u = rand_links(L, np.random.default_rng(51), beta=2.0)
    with thirring.Lattice(*dims, kernel=1) as G:
        G.set_links(u)
        G.init_random(987654321.0)
        got = G.measure(1e-8, 0.1, 1, kernel_meas=1, knoise=3)
    return (np.asarray(got["parts"], dtype=np.float64).tobytes().hex(),
            [int(v) for v in got["itercg"]], float(got["psibarpsi"]))


@pytest.mark.gpu
def test_measure_same_bits_in_fresh_processes():
    # the batched FP64 measurement solves have no run-dependent choice: two fresh
    # processes (each tuning its stencils anew) give identical bits
    import os
    import subprocess
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    code = ("import sys, json; sys.path.insert(0, %r); import conftest; import test_measure_gpu as t; "
            "print(json.dumps(t._measure_bits()))" % here)
    outs = []
    for _ in range(2):
        r = subprocess.run([sys.executable, "-c", code], cwd=here, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        outs.append(r.stdout.strip().splitlines()[-1])
    assert outs[0] == outs[1]
