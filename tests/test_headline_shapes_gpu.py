"""Parity at the shapes the benchmarks time (dirac.F90, multishift_module.F90).

The stencil tests elsewhere use small lattices and Ls <= 24.  Here the FP64
operators run where the timed kernels run: Ls = 32 (a site's 32 threads are a
whole warp, fifth-dimension neighbours by shuffle), Ls = 48 (neighbours by
load), the smallest and a middle config-2 lattice, and the fused epilogues
of the solvers (out = aux + c Op in, out = Op in + c aux, with |out|^2).
Tolerances: FP64 1e-13 relative to max|oracle|, FP32
storage 2e-6; the epilogue norms to 1e-12 relative.
"""
import os

import numpy as np
import pytest

import oracle as O
import thirring
from helpers import interior, rand_links, rand_spinor, rel_err

TOL = 1e-13
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.gpu
@pytest.mark.parametrize("dims,kernel,imasses", [
    ((16, 16, 16, 16), 0, (1, 3, 5)),
    ((16, 16, 16, 32), 0, (1, 3, 5)),
    ((16, 16, 16, 48), 0, (1, 3, 5)),
    ((16, 16, 16, 32), 1, (1, 3)),
    ((24, 24, 24, 16), 0, (3,)),
    ((32, 32, 32, 32), 0, (1,)),
])
def test_dslash_fp64_headline_shapes(dims, kernel, imasses):
    rng = np.random.default_rng(sum(dims) + 7 * kernel)
    L = O.lat(*dims, kernel=kernel)
    u = rand_links(L, rng, beta=0.3)
    R = rand_spinor(L, rng)
    with thirring.Lattice(*dims, kernel=kernel) as G:
        G.set_links(u)
        for imass in imasses:
            for dag in (False, True):
                ref = (O.dslashd if dag else O.dslash)(L, R, u, 0.01, imass)
                got = (G.dslashd if dag else G.dslash)(R, None, 0.01, imass)
                e = rel_err(interior(got), interior(ref))
                assert e <= TOL, (dims, kernel, imass, dag, e)


def _epilogue_ref(L, u, R, aux, coef, am, imass, dag, mode):
    op = interior((O.dslashd if dag else O.dslash)(L, R, u, am, imass))
    if mode == 0:
        out = op
    elif mode == 1:
        out = interior(aux) + coef * op
    else:
        out = op + coef * interior(aux)
    return out, float(np.sum(np.abs(out) ** 2))


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(8, 8, 8, 32), (16, 16, 16, 32), (8, 8, 4, 48)])
@pytest.mark.parametrize("precision", [0, 2, 3])
def test_fused_epilogues(dims, precision):
    """The epilogues the solvers run (congrad: |M p|^2 and r - alpha M^dagger x1;
    batched multishift: h = M r + gamma h and r + omega M^dagger h) at Ls = 32 and 48,
    FP64, FP32 and BF16 storage, against the oracle's operator composed on the host.
    BF16 keeps 8 significant bits: inputs and output each round by up to 2^-9
    relative, FP32 arithmetic in between.  The same roundings emulated on the host
    on these cases give at most 4.4e-3 (max-norm relative) and 5.8e-5 on |out|^2,
    so the bounds are 1e-2 and 1e-3."""
    rng = np.random.default_rng(sum(dims) + precision)
    L = O.lat(*dims)
    u = rand_links(L, rng, beta=0.3)
    R, aux = rand_spinor(L, rng), rand_spinor(L, rng)
    tol = {0: TOL, 2: 2e-6, 3: 1e-2}[precision]
    with thirring.Lattice(*dims) as G:
        G.set_links(u)
        for imass in (1, 3, 5):
            for mode, dag, coef in ((0, False, 0.0), (3, False, 0.61), (1, True, -0.37), (1, False, 1.25),
                                    (3, True, -2.0)):
                ref, n2_ref = _epilogue_ref(L, u, R, aux, coef, 0.01, imass, dag, mode)
                got, n2 = G.dslash_fused(R, aux if mode else None, coef, 0.01, imass, dag, mode, precision)
                e = rel_err(interior(got), ref)
                assert e <= tol, (imass, mode, dag, e)
                n2_tol = {0: 1e-12, 2: 1e-5, 3: 1e-3}[precision]
                assert abs(n2 - n2_ref) <= n2_tol * n2_ref, (imass, mode, dag)


@pytest.mark.gpu
def test_multishift_25_poles_remez4_per_shift():
    """The batched FP64 multishift with remez4's 25 poles (shifts 7.8e-6 .. 1.2e3) on a
    12^2 x 12, Ls 16 lattice at beta 0.3, am 0.01, res 1e-9 against the oracle
    (multishift_module.F90:13-284): iteration counts within 2 or 0.5 % (about 5500 here:
    sums taken in another order move the exit by a few iterations), and for every shift the
    true residual |input - (M^dagger M + aden_k) x_k| times correction_k (the
    quantity :244 tests on the recursive residual) no worse than twice the oracle's
    own or res, and the solution equal to the oracle's to 1e-7 relative."""
    rng = np.random.default_rng(2024)
    L = O.lat(12, 12, 12, 16)
    u = rand_links(L, rng, beta=0.3)
    inp = rand_spinor(L, rng) / np.sqrt(2)
    an, ad, _, _ = O.read_remez(os.path.join(GOLD, "remez4"), 25)
    anum, res = an[1:], 1e-9
    out_ref, it_ref, cgr_ref = O.multishift(L, u, 0.01, 1, anum, ad, inp, res, 50000)
    with thirring.Lattice(12, 12, 12, 16) as G:
        G.set_links(u)
        out, it, cgr = G.multishift_solver(None, 0.01, 1, ad, anum, inp, res, 50000)
        r2 = G.shift_residuals(inp, out, ad, 0.01, 1)
        r2_ref = G.shift_residuals(inp, out_ref, ad, 0.01, 1)
        # the mixed multishift (qmrherm iflag 1 returns its shifted solutions in Phi0)
        Phi0 = np.zeros(G.sshape + (G.ndiag,), np.complex128, order="F")
        _, it_m, _ = G.qmrherm(inp, res, 0.01, 1, an, ad, 1, use_sp=thirring.MIXED_FP32, Phi0=Phi0)
        sw = G.mixed_switched_at()
        out_m = np.asfortranarray(Phi0[1:-1, 1:-1, 1:-1, 1:-1, :, :25])
        r2_m = G.shift_residuals(inp, out_m, ad, 0.01, 1)
    corr = np.abs(anum / ad)
    corr = corr / np.exp(np.mean(np.log(corr)))
    tr, tr_ref = np.sqrt(r2) * corr, np.sqrt(r2_ref) * corr
    err = np.array([np.linalg.norm(out[..., k] - out_ref[..., k]) / np.linalg.norm(out_ref[..., k])
                    for k in range(25)])
    print("iterations", it, it_ref)
    print("true residual * correction / res (GPU):   ", " ".join("%.2g" % v for v in tr / res))
    print("true residual * correction / res (oracle):", " ".join("%.2g" % v for v in tr_ref / res))
    print("relative error vs oracle:", " ".join("%.1g" % v for v in err))
    tol = max(2, it_ref // 200)
    assert abs(it - it_ref) <= tol and np.max(np.abs(cgr - cgr_ref)) <= tol
    assert np.all(tr <= 2 * np.maximum(tr_ref, res)), tr / np.maximum(tr_ref, res)
    assert np.max(err) <= 1e-7, err
    assert np.all(out[..., 25:] == 0)
    # mixed precision: the same bars against the FP64 oracle
    tr_m = np.sqrt(r2_m) * corr
    err_m = np.array([np.linalg.norm(out_m[..., k] - out_ref[..., k]) / np.linalg.norm(out_ref[..., k])
                      for k in range(25)])
    print("mixed: iterations %d, left FP64 at %d" % (it_m, sw))
    print("true residual * correction / res (mixed): ", " ".join("%.2g" % v for v in tr_m / res))
    print("relative error vs oracle (mixed):", " ".join("%.1g" % v for v in err_m))
    assert 0 < sw < it_m and abs(it_m - it_ref) <= tol
    assert np.all(tr_m <= 2 * np.maximum(tr_ref, res)), tr_m / np.maximum(tr_ref, res)
    assert np.max(err_m) <= 1e-7, err_m
