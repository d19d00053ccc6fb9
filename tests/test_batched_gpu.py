"""Batched measurement solves vs the oracle's congrad (measure_module.F90:9-140).

Each right-hand side / packed lattice must meet congrad's rule on its FP64
true residual, |b - M^dagger M x|^2 < 4 V Ls res^2, in every precision mode,
and agree with the oracle's solution (same problem) within the amplification
that CG rounding allows on these small ill-conditioned lattices.
"""
import numpy as np
import pytest

import oracle as O
import thirring
from helpers import interior, rand_links, rand_spinor, rel_err

MODES = [0, 2, 3]  # FP64, mixed FP32, mixed BF16


def _true_r2(L, u, b, x, am, imass):
    return float(np.sum(np.abs(interior(b) - interior(O.dirac_operator(L, x, u, am, imass))) ** 2))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", MODES)
@pytest.mark.parametrize("kernel", [0, 1])
def test_congrad_multi(precision, kernel):
    rng = np.random.default_rng(31 + precision + 10 * kernel)
    dims = (4, 4, 6, 8)
    L = O.lat(*dims, kernel=kernel)
    u = rand_links(L, rng, beta=2.0)
    nrhs = 5
    Phi = np.stack([rand_spinor(L, rng) for _ in range(nrhs)], axis=-1)
    Phi = np.asfortranarray(Phi)
    X = np.zeros_like(Phi)
    # smooth links (theta width 1/sqrt(2)) keep every precision mode far inside
    # congrad's cap niterc = Ls*V3: the FP64 oracle needs 155 (Shamir) / 238 (Wilson) of 768
    res, am, imass = 1e-8, 0.1, 3
    with thirring.Lattice(*dims, kernel=kernel) as G:
        G.set_links(u)
        its, outer = G.congrad_multi(Phi, X, res, am, imass, precision)
    resid = 4 * 4 * 4 * 6 * 8 * res * res
    for k in range(nrhs):
        xr = O.spinor(L)
        O.congrad(L, np.asfortranarray(Phi[..., k]), xr, u, res, am, imass)
        xk = np.asfortranarray(X[..., k])
        O.update_halo_5(L, xk)
        assert _true_r2(L, u, Phi[..., k], xk, am, imass) < resid, (k, its[k])
        assert rel_err(interior(xk), interior(xr)) <= 1e-5
    if precision != 0:
        assert outer >= 1


@pytest.mark.gpu
def test_congrad_multi_reference_kat():
    # tests/test_congrad.F90 fixture through the batched path: itercg == 27 for every copy
    L = O.lat(12, 12, 12, 24)
    st = O.starting_state(L, X=True)
    Phi = np.asfortranarray(np.stack([st["Phi"]] * 3, axis=-1))
    X = np.asfortranarray(np.stack([st["X"]] * 3, axis=-1))
    X_ref = st["X"].copy(order="F")
    O.congrad(L, st["Phi"], X_ref, st["u"], 0.1, 0.05, 3)
    with thirring.Lattice(12, 12, 12, 24) as G:
        G.set_links(st["u"])
        its, _ = G.congrad_multi(Phi, X, 0.1, 0.05, 3, 0)
    assert list(its) == [27, 27, 27]
    for k in range(3):
        assert rel_err(interior(np.asfortranarray(X[..., k])), interior(X_ref)) <= 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("precision", MODES)
def test_packed_uneven_lattices(precision):
    rng = np.random.default_rng(77 + precision)
    shapes = [(4, 4, 4, 8), (6, 6, 6, 4), (4, 6, 8, 12), (8, 8, 8, 8)]
    # smooth links keep every lattice far inside its cap niterc = Ls*V3 in all modes
    res, am, imass = 1e-8, 0.5, 1
    pack = thirring.Pack(shapes)
    lats, us, phis = [], [], []
    for i, (lx, ly, lt, ls) in enumerate(shapes):
        L = O.lat(lx, ly, lt, ls, beta=0.3 + 0.05 * i)
        u = rand_links(L, rng, beta=2.0 + 0.5 * i)
        phi = rand_spinor(L, rng)
        pack.upload(i, u, phi, O.spinor(L))
        lats.append(L); us.append(u); phis.append(phi)
    its, outer = pack.congrad(res, am, imass, precision)
    for i, L in enumerate(lats):
        x = pack.download(i)
        resid = 4 * L.lx * L.ly * L.lt * L.ls * res * res
        assert _true_r2(L, us[i], phis[i], x, am, imass) < resid, (i, its[i])
        xr = O.spinor(L)
        O.congrad(L, phis[i], xr, us[i], res, am, imass)
        assert rel_err(interior(x), interior(xr)) <= 1e-5
    pack.close()
