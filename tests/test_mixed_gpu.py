"""The mixed-precision multishift (qmrherm use_sp = THR_MIXED_FP32 / _BF16).

The solve runs in FP64 until the base residual falls below a fraction of
|Phi| and then continues with the stencils, residuals and search direction in
FP32 (or BF16 storage with FP32 arithmetic); the shifted solutions stay FP64.
Criterion, per shift: the true residual |Phi - (M^dagger M + aden_k) x_k|
times the reference's correction_k (multishift_module.F90:87-88, :244) is no
worse than twice the FP64 solve's own (or res), and the solution equals the
FP64 solve's to 1e-9 relative.  Poles: 25, log-spaced 1e-5 .. 1e2 with
x^-1/2 residues (the benchmark's rational function).
"""
import numpy as np
import pytest

import oracle as O
import thirring
from helpers import rand_links, rand_spinor


def rational(n=25):
    s = np.logspace(-5.0, 2.0, n)
    a = np.sqrt(s) * (7.0 / (n - 1)) * np.log(10.0) / np.pi
    return np.concatenate([[0.0], a]), s


def _solve(G, phi, mode, anum, aden, res=1e-9):
    Phi0 = np.zeros(G.sshape + (G.ndiag,), np.complex128, order="F")  # iflag 1 returns the shifted solutions
    x, it, cgr = G.qmrherm(phi, res, 0.01, 1, anum, aden, 1, use_sp=mode, Phi0=Phi0)
    shifts = np.asfortranarray(Phi0[1:-1, 1:-1, 1:-1, 1:-1, :, :len(aden)])
    return x, it, shifts, G.mixed_switched_at()


@pytest.mark.gpu
@pytest.mark.parametrize("mode,switch", [(thirring.MIXED_FP32, 1e-8), (thirring.MIXED_BF16, 1e-13)])
def test_mixed_multishift_matches_fp64(mode, switch):
    rng = np.random.default_rng(77)
    dims = (12, 12, 12, 16)
    L = O.lat(*dims)
    u = rand_links(L, rng, beta=0.3)
    phi = rand_spinor(L, rng) / np.sqrt(2)
    anum, aden = rational()
    corr = np.abs(anum[1:] / aden)
    corr = corr / np.exp(np.mean(np.log(corr)))
    with thirring.Lattice(*dims) as G:
        G.set_links(u)
        G.set_mixed(switch, switch)
        x64, it64, s64, sw64 = _solve(G, phi, 0, anum, aden)
        xm, itm, sm, swm = _solve(G, phi, mode, anum, aden)
        tr64 = np.sqrt(G.shift_residuals(phi, s64, aden, 0.01, 1)) * corr
        trm = np.sqrt(G.shift_residuals(phi, sm, aden, 0.01, 1)) * corr
    err = np.array([np.linalg.norm(sm[..., k] - s64[..., k]) / np.linalg.norm(s64[..., k]) for k in range(25)])
    print("iterations fp64 %d mixed %d, left FP64 at %d" % (it64, itm, swm))
    print("true residual * correction / res, fp64: ", " ".join("%.2g" % v for v in tr64 / 1e-9))
    print("true residual * correction / res, mixed:", " ".join("%.2g" % v for v in trm / 1e-9))
    print("relative error vs fp64:", " ".join("%.1g" % v for v in err))
    assert sw64 == 0
    if mode == thirring.MIXED_FP32:
        assert 0 < swm < itm  # the FP32 phase ran
    assert abs(itm - it64) <= max(2, it64 // 100)
    assert np.all(trm <= 2 * np.maximum(tr64, 1e-9)), trm / np.maximum(tr64, 1e-9)
    assert np.max(err) <= 1e-9, err
    assert np.max(np.abs(xm - x64)) <= 1e-9 * np.max(np.abs(x64))


@pytest.mark.gpu
def test_mixed_multishift_graph_equals_host_launched():
    """The precision switch happens between the same two batches whether the loop
    runs as a CUDA graph or is launched batch by batch from the host."""
    rng = np.random.default_rng(5)
    dims = (8, 8, 8, 8)
    L = O.lat(*dims)
    u = rand_links(L, rng, beta=0.5)
    phi = rand_spinor(L, rng)
    anum, aden = rational()
    outs = []
    with thirring.Lattice(*dims) as G:
        G.set_links(u)
        G.set_mixed(1e-5, 1e-5)
        for algo in (1, 2, 1):
            G.set_solver(algo)
            for mode in (thirring.MIXED_FP32, thirring.MIXED_BF16):
                x, it, cgr = G.qmrherm(phi, 1e-9, 0.01, 1, anum, aden, 0, use_sp=mode)
                outs.append((algo, mode, x, it, G.mixed_switched_at()))
    for (a0, m0, x0, i0, s0) in outs[:2]:
        assert s0 > 0
        for (a, m, x, i, s) in outs[2:]:
            if m == m0:
                assert (i, s) == (i0, s0) and np.array_equal(x, x0), (a, m)
