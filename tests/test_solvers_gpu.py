"""congrad, multishift_solver(_sp), qmrherm and derivs on the GPU vs the oracle.

Short solves (the reference's own fixtures: a few iterations) must agree with
the oracle to 1e-10 or better.  Long solves (hundreds to thousands of CG
iterations on random ill-conditioned lattices) amplify FP64 rounding
differences, so there the criterion is the reference's: the same iteration
count within 2, and a true residual that meets the stopping rule; solutions
then agree to ~1e-6 relative.  The single-precision reference solver
(multishift_solver_sp) agrees to 1e-4.
"""
import os

import numpy as np
import pytest

import oracle as O
import thirring
from helpers import interior, rand_links, rand_spinor, rel_err

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def remez(name, n):
    return O.read_remez(os.path.join(GOLD, name), n)  # (anumA, adenA, anumB, adenB)


@pytest.mark.gpu
def test_congrad_kat_and_parity():
    # tests/test_congrad.F90: itercg == 27 on the 12^3 x 24 analytic state
    L = O.lat(12, 12, 12, 24)
    st = O.starting_state(L, X=True)
    X_ref = st["X"].copy(order="F")
    it_ref, _ = O.congrad(L, st["Phi"], X_ref, st["u"], 0.1, 0.05, 3)
    with thirring.Lattice(12, 12, 12, 24) as G:
        G.set_links(st["u"])
        X = st["X"].copy(order="F")
        itercg, nx = G.congrad(st["Phi"], X, 0.1, 0.05, 3)
    assert itercg == 27 == it_ref and nx == 27
    assert rel_err(interior(X), interior(X_ref)) <= 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("kernel,imass,layout", [(0, 1, 0), (0, 3, 1), (0, 5, 0), (1, 1, 0), (1, 3, 1)])
def test_congrad_tight(kernel, imass, layout):
    rng = np.random.default_rng(11 + kernel + imass)
    L = O.lat(4, 4, 6, 8, kernel=kernel)
    u = rand_links(L, rng)
    Phi = rand_spinor(L, rng)
    X_ref = O.spinor(L)
    it_ref, _ = O.congrad(L, Phi, X_ref, u, 1e-9, 0.05, imass)
    with thirring.Lattice(4, 4, 6, 8, kernel=kernel, layout=layout) as G:
        G.set_links(u)
        X = O.spinor(L)
        it, _ = G.congrad(Phi, X, 1e-9, 0.05, imass)
    assert abs(it - it_ref) <= 2
    assert rel_err(interior(X), interior(X_ref)) <= 1e-4
    # CG's recursive residual meets |r|^2 < 4 V Ls res^2; on these ill-conditioned random
    # lattices the true residual drifts above it in the oracle too: compare the two
    r = np.linalg.norm(interior(Phi) - interior(O.dirac_operator(L, X, u, 0.05, imass)))
    r_ref = np.linalg.norm(interior(Phi) - interior(O.dirac_operator(L, X_ref, u, 0.05, imass)))
    assert r <= 3 * r_ref + 10 * np.sqrt(4 * 4 * 4 * 6 * 8) * 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("sp", [False, True])
def test_multishift_vs_oracle(sp):
    rng = np.random.default_rng(3)
    L = O.lat(4, 4, 4, 8)
    u = rand_links(L, rng)
    inp = rand_spinor(L, rng)
    an, ad, _, _ = remez("remez2g", 12)
    res = 1e-6 if sp else 1e-9
    out_ref, it_ref, cgr_ref = O.multishift(L, u, 0.05, 1, an[1:], ad, inp, res, 5000, sp=sp)
    with thirring.Lattice(4, 4, 4, 8) as G:
        out, it, cgr = G.multishift_solver(u, 0.05, 1, ad, an[1:], inp, res, 5000, sp=sp)
    if sp:
        assert abs(it - it_ref) <= 3
        assert rel_err(out[..., :12], out_ref[..., :12]) <= 1e-4
    else:
        assert abs(it - it_ref) <= 2 and np.max(np.abs(cgr - cgr_ref)) <= 2
        assert rel_err(out[..., :12], out_ref[..., :12]) <= 1e-5
        # every shifted system meets the reference's stopping rule |r_i| * correction_i < res
        corr = np.abs(an[1:] / ad)
        corr = corr / np.exp(np.mean(np.log(corr)))
        for k in range(12):
            xk = O.spinor(L)
            xk[1:-1, 1:-1, 1:-1, 1:-1, :] = out[..., k]
            O.update_halo_5(L, xk)
            r = interior(inp) - interior(O.dirac_operator(L, xk, u, 0.05, 1)) - ad[k] * interior(xk)
            assert np.linalg.norm(r) * corr[k] < 10 * res, k
    assert np.all(out[..., 12:] == 0)


@pytest.mark.gpu
@pytest.mark.parametrize("sp", [False, True])
def test_multishift_batched_equals_per_iteration(sp):
    """The batched shift update replays the reference's per-iteration updates."""
    rng = np.random.default_rng(8)
    L = O.lat(4, 4, 6, 8)
    u = rand_links(L, rng)
    inp = rand_spinor(L, rng)
    an, ad, _, _ = remez("remez4g", 12)
    res = 1e-6 if sp else 1e-9
    outs = []
    with thirring.Lattice(4, 4, 6, 8) as G:
        for algo in (0, 1):
            G.set_solver(algo)
            outs.append(G.multishift_solver(u, 0.05, 3, ad, an[1:], inp, res, 5000, sp=sp))
    (o0, i0, c0), (o1, i1, c1) = outs
    assert abs(i0 - i1) <= 2 and np.max(np.abs(c0 - c1)) <= 2
    assert rel_err(o1[..., :12], o0[..., :12]) <= (1e-4 if sp else 1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", [0, 1])
def test_qmrherm_all_iflags(kernel):
    rng = np.random.default_rng(17 + kernel)
    L = O.lat(4, 4, 6, 8, kernel=kernel)
    u = rand_links(L, rng)
    Phi = rand_spinor(L, rng)
    an, ad, _, _ = remez("remez4g", 12)
    Phi0_ref = np.zeros((L.ls + 2, L.lx + 2, L.ly + 2, L.lt + 2, 4, 25), np.complex128, order="F")
    dS_ref = O.field3(L)
    with thirring.Lattice(4, 4, 6, 8, kernel=kernel) as G:
        G.set_links(u)
        Phi0 = np.zeros_like(Phi0_ref)
        dS = O.field3(L)
        for iflag in (0, 1, 2, 3):
            x_ref, it_ref, _, rc = O.qmrherm(L, u, Phi, 1e-9, 0.05, 3, an, ad, iflag, dSdpi=dS_ref, Phi0=Phi0_ref)
            assert rc == 0
            x, it, _ = G.qmrherm(Phi, 1e-9, 0.05, 3, an, ad, iflag, dSdpi=dS, Phi0=Phi0)
            assert abs(it - it_ref) <= max(2, it_ref // 200)
            assert rel_err(interior(x), interior(x_ref)) <= 1e-6, iflag
            if iflag == 1:
                assert rel_err(Phi0[1:-1, 1:-1, 1:-1, 1:-1, :, :12], Phi0_ref[1:-1, 1:-1, 1:-1, 1:-1, :, :12]) <= 1e-5
            if iflag >= 2:
                assert rel_err(dS, dS_ref) <= 1e-5, iflag


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", [0, 1])
def test_qmrherm_reference_fixture(kernel):
    """tests/test_qmrherm.F90 with tests/test_params.F90:55 (max_qmr_iters = 2):
    12^3 x 24 analytic state, res 0.1, am 0.05, imass 3, anum(i) = Re exp(i i tau/25),
    aden(i) = Re exp(-i 0.5 i tau/25), Phi0 reset to the fixture before every call;
    the reference asserts itercg == 2."""
    L = O.lat(12, 12, 12, 24, kernel=kernel)
    tau = 8 * np.arctan(1.0)
    i = np.arange(1, 26)
    anum = np.concatenate([[0.5], np.cos(i * tau / 25)])
    aden = np.cos(0.5 * i * tau / 25)
    st = O.starting_state(L, Phi0=True)
    dS_ref = O.field3(L)
    dS = O.field3(L)
    with thirring.Lattice(12, 12, 12, 24, kernel=kernel) as G:
        G.set_links(st["u"])
        for iflag in range(4):
            P_ref = st["Phi0"].copy(order="F")
            P = st["Phi0"].copy(order="F")
            x_ref, it_ref, _, rc = O.qmrherm(L, st["u"], st["Phi"], 0.1, 0.05, 3, anum, aden, iflag, max_iters=2,
                                            dSdpi=dS_ref, Phi0=P_ref)
            x, it, _ = G.qmrherm(st["Phi"], 0.1, 0.05, 3, anum, aden, iflag, dSdpi=dS, Phi0=P, max_qmr_iters=2)
            assert it == it_ref == 2
            assert rel_err(interior(x), interior(x_ref)) <= 1e-11
            assert rel_err(P[1:-1, 1:-1, 1:-1, 1:-1], P_ref[1:-1, 1:-1, 1:-1, 1:-1]) <= 1e-11
            assert rel_err(dS, dS_ref) <= 1e-11


@pytest.mark.gpu
def test_qmrherm_guards():
    # qmrherm_module.F90:66-81: ndiagq > ndiag and Ls % 4 != 0 abort the reference
    rng = np.random.default_rng(4)
    L = O.lat(4, 4, 4, 6)
    Phi = rand_spinor(L, rng)
    an, ad, _, _ = remez("remez4g", 12)
    with thirring.Lattice(4, 4, 4, 6) as G:
        G.coef(np.zeros((4, 4, 4, 3), np.float32))
        with pytest.raises(thirring.ThirringError) as e:
            G.qmrherm(Phi, 1e-6, 0.05, 1, an, ad, 0)
        assert e.value.status == 2


@pytest.mark.gpu
@pytest.mark.parametrize("kernel,iflag,imass", [(0, 0, 1), (0, 1, 3), (1, 0, 1), (1, 1, 3), (1, 0, 3), (1, 1, 1)])
def test_derivs_vs_oracle(kernel, iflag, imass):
    rng = np.random.default_rng(100 + 10 * kernel + iflag)
    L = O.lat(4, 6, 4, 8, kernel=kernel)
    R, X2 = rand_spinor(L, rng), rand_spinor(L, rng)
    dS0 = np.asfortranarray(rng.standard_normal((4, 6, 4, 3)))
    ref = O.derivs(L, R, X2, 0.37, iflag, 0.05, imass, dS0.copy(order="F"))
    with thirring.Lattice(4, 6, 4, 8, kernel=kernel) as G:
        got = G.derivs(R, X2, 0.37, iflag, 0.05, imass, dS0.copy(order="F"))
    assert rel_err(got, ref) <= 1e-12


@pytest.mark.gpu
def test_derivs_reference_fixture():
    # tests/test_derivs_shamir.F90: anum = tau, iflag 0, imass 3, am 0.05, dSdpi = fixture
    L = O.lat(12, 12, 12, 24)
    st = O.starting_state(L, R=True, X=True, dSdpi=True)
    tau = 8 * np.arctan(1.0)
    ref = O.derivs(L, st["R"], st["X"], tau, 0, 0.05, 3, st["dSdpi"].copy(order="F"))
    with thirring.Lattice(12, 12, 12, 24) as G:
        got = G.derivs(st["R"], st["X"], tau, 0, 0.05, 3, st["dSdpi"].copy(order="F"))
    assert rel_err(got, ref) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("sp", [False, True])
@pytest.mark.parametrize("maxcg", [5000, 21])
def test_multishift_graph_equals_host_launched(sp, maxcg):
    """The graph-driven batch loop (WHILE node) runs exactly the kernels of the
    host-launched loop: identical results, also when the iteration cap ends it."""
    rng = np.random.default_rng(12)
    L = O.lat(4, 4, 6, 8)
    u = rand_links(L, rng)
    inp = rand_spinor(L, rng)
    an, ad, _, _ = remez("remez4g", 12)
    res = 1e-6 if sp else 1e-9
    outs = []
    with thirring.Lattice(4, 4, 6, 8) as G:
        for algo in (1, 2, 1):  # graph, host-launched, graph again (cached graph)
            G.set_solver(algo)
            outs.append(G.multishift_solver(u, 0.05, 3, ad, an[1:], inp, res, maxcg, sp=sp))
    for o, it, cgr in outs[1:]:
        assert it == outs[0][1] and np.array_equal(cgr, outs[0][2])
        assert np.array_equal(o, outs[0][0])
    if maxcg == 21:
        assert outs[0][1] == 21


@pytest.mark.gpu
def test_congrad_graph_equals_host_launched():
    """congrad's chunk loop as a CUDA graph gives the bits of the host-launched loop."""
    rng = np.random.default_rng(21)
    L = O.lat(4, 4, 6, 8)
    u = rand_links(L, rng, beta=2.0)
    Phi = rand_spinor(L, rng)
    outs = []
    with thirring.Lattice(4, 4, 6, 8) as G:
        G.set_links(u)
        for algo in (1, 2, 1):
            G.set_solver(algo)
            X = O.spinor(L)
            it, nx = G.congrad(Phi, X, 1e-9, 0.1, 3)
            outs.append((it, nx, X))
    for it, nx, X in outs[1:]:
        assert (it, nx) == outs[0][:2] and np.array_equal(X, outs[0][2])


@pytest.mark.gpu
@pytest.mark.parametrize("env", [{"THR_OVERLAP": "0"}, {"THR_REVERSE": "1"}, {"THR_REVERSE": "0"},
                                 {"THR_GRAPHS": "0"}, {"THR_PDL": "0"}, {"THR_CHAIN": "1"}])
def test_solver_schedules_bit_identical(tmp_path, env):
    """Where the batched multishift's flush runs (side stream or in line), which
    way the solver kernels sweep the sites, whether the loops are graphs or
    host-launched, whether the kernel chain uses dependent launches, and whether a
    batch runs as the kernel chain or as one persistent kernel (THR_CHAIN=1: this
    lattice is small enough for it) change the schedule only: the multishift (FP64 and
    FP32 vectors) and congrad give the same bits and iteration counts."""
    import os
    import subprocess
    import sys
    rng = np.random.default_rng(31)
    L = O.lat(4, 4, 6, 8)
    u = rand_links(L, rng)
    inp = rand_spinor(L, rng)
    an, ad, _, _ = remez("remez4g", 12)
    np.savez(tmp_path / "in.npz", u=u, inp=inp, an=an, ad=ad)
    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "thirring-rhmc_b200")
    code = ("import sys, numpy as np; sys.path.insert(0, %r); import thirring; d = %r; t = sys.argv[1];"
            "z = np.load(d + '/in.npz'); u = np.asfortranarray(z['u']); inp = np.asfortranarray(z['inp']);"
            "G = thirring.Lattice(4, 4, 6, 8); r = {};"
            "r['x64'], r['i64'], r['c64'] = G.multishift_solver(u, 0.05, 3, z['ad'], z['an'][1:], inp, 1e-9, 5000);"
            "r['x32'], r['i32'], r['c32'] = G.multishift_solver(u, 0.05, 3, z['ad'], z['an'][1:], inp, 1e-6, 5000,"
            " sp=True);"
            "G.set_links(u); X = np.zeros_like(inp); r['icg'], _ = G.congrad(inp, X, 1e-9, 0.05, 3); r['xcg'] = X;"
            "np.savez(d + '/out_' + t + '.npz', **r); G.close()" % (pkg, str(tmp_path)))
    subprocess.run([sys.executable, "-c", code, "ref"], check=True)
    subprocess.run([sys.executable, "-c", code, "alt"], check=True, env=dict(os.environ, **env))
    ref, got = np.load(tmp_path / "out_ref.npz"), np.load(tmp_path / "out_alt.npz")
    for k in ref.files:
        assert np.array_equal(ref[k], got[k]), k


def _chain_run(tmp_path, dims, tag, env, poles=12, res=1e-9):
    """A batched FP64 multishift (remez4g's poles) in a fresh process; returns its
    exit status, output and the solve's status code (0 or the ThirringError's)."""
    import os
    import subprocess
    import sys
    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "thirring-rhmc_b200")
    code = ("import sys, numpy as np; sys.path.insert(0, %r); import thirring; d = %r; t = sys.argv[1];"
            "z = np.load(d + '/in.npz'); u = np.asfortranarray(z['u']); inp = np.asfortranarray(z['inp']);"
            "G = thirring.Lattice(*%r); r = {'status': 0};"
            "\ntry:\n r['x'], r['i'], r['c'] = G.multishift_solver(u, 0.05, 3, z['ad'], z['an'][1:], inp, %r, 20000)"
            "\nexcept thirring.ThirringError as e:\n r['status'] = e.status"
            "\nG.close(); np.savez(d + '/out_' + t + '.npz', **r)" % (pkg, str(tmp_path), dims, res))
    r = subprocess.run([sys.executable, "-c", code, tag], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, **env))
    assert r.returncode == 0, r.stdout + r.stderr
    return np.load(tmp_path / ("out_%s.npz" % tag))


@pytest.mark.gpu
def test_chain_several_site_blocks_per_block(tmp_path):
    """The persistent multishift kernel forced (THR_CHAIN=2) on a lattice with more
    stencil site blocks than resident blocks (24^3, Ls 16: 1728 site blocks), so each
    block walks several of them between two barriers: the same bits and iteration
    counts as the kernel chain (THR_CHAIN=0)."""
    rng = np.random.default_rng(41)
    dims = (24, 24, 24, 16)
    L = O.lat(*dims)
    an, ad, _, _ = remez("remez4g", 12)
    np.savez(tmp_path / "in.npz", u=rand_links(L, rng), inp=rand_spinor(L, rng), an=an, ad=ad)
    a = _chain_run(tmp_path, dims, "chain", {"THR_CHAIN": "2"}, res=1e-7)
    b = _chain_run(tmp_path, dims, "plain", {"THR_CHAIN": "0"}, res=1e-7)
    assert int(a["status"]) == 0 and int(b["status"]) == 0
    for k in ("x", "i", "c"):
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.gpu
def test_chain_barrier_timeout(tmp_path):
    """The persistent multishift kernel's bounded grid barriers (THR_CHAIN=1).  With
    THR_CHAIN_WAIT_TEST=1 every barrier waits for one arrival more than the grid
    has, so each wait runs out after 0.2 s (nothing faults and nothing is left
    waiting on the GPU): the solve ends with THR_ERR_TIMEOUT (8).  The same solve
    in a fresh process without the test switch converges and matches the oracle."""
    rng = np.random.default_rng(43)
    dims = (4, 4, 6, 8)
    L = O.lat(*dims)
    u, inp = rand_links(L, rng), rand_spinor(L, rng)
    an, ad, _, _ = remez("remez4g", 12)
    np.savez(tmp_path / "in.npz", u=u, inp=inp, an=an, ad=ad)
    bad = _chain_run(tmp_path, dims, "bound", {"THR_CHAIN": "1", "THR_CHAIN_WAIT_TEST": "1"})
    assert int(bad["status"]) == 8
    good = _chain_run(tmp_path, dims, "ok", {"THR_CHAIN": "1"})
    assert int(good["status"]) == 0
    ref, it_ref, _ = O.multishift(L, u, 0.05, 3, an[1:], ad, inp, 1e-9, 20000)
    assert abs(int(good["i"]) - it_ref) <= 2
    assert rel_err(good["x"][..., :12], ref[..., :12]) <= 1e-5
