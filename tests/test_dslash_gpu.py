"""dslash / dslashd on the GPU against the oracle (dirac.F90).

FP64 tolerance: max|GPU - oracle| <= 1e-13 * max|oracle|.
Also: the even-odd storage order gives bit-identical results to the natural
one, and M^dagger is the adjoint of M.
"""
import numpy as np
import pytest

import oracle as O
import thirring
from helpers import interior, rand_links, rand_spinor, rel_err

TOL = 1e-13

CASES = [(k, im, lay) for k in (0, 1) for im in ((1, 3, 5) if k == 0 else (1, 3)) for lay in (0, 1)]


@pytest.mark.gpu
@pytest.mark.parametrize("kernel,imass,layout", CASES)
@pytest.mark.parametrize("dims", [(4, 6, 8, 8), (6, 4, 4, 12), (4, 4, 6, 8), (8, 4, 2, 16)])
def test_dslash_random(kernel, imass, layout, dims):
    """The last two shapes are ones the staged-tile FP64 Shamir kernel (THR_TILE=1)
    takes in the natural site order (Lx, Ly multiples of 4, Lt of 2, Ls of 8);
    by default they run on k_dslash like the first two."""
    rng = np.random.default_rng(hash((kernel, imass, layout) + dims) % 2**32)
    lx, ly, lt, ls = dims
    L = O.lat(lx, ly, lt, ls, kernel=kernel, am3=1.0)
    u = rand_links(L, rng)
    R = rand_spinor(L, rng)
    with thirring.Lattice(lx, ly, lt, ls, kernel=kernel, layout=layout) as G:
        for dag in (False, True):
            ref = (O.dslashd if dag else O.dslash)(L, R, u, 0.01, imass)
            got = (G.dslashd if dag else G.dslash)(R, u, 0.01, imass)
            e = rel_err(interior(got), interior(ref))
            assert e <= TOL, (dag, e)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel,imass", [(0, 1), (0, 3), (0, 5), (1, 1), (1, 3)])
def test_dslash_reference_fixture(kernel, imass):
    # tests/test_dslash_shamir.F90: 12^3 x 24 analytic state, am = 0.05
    L = O.lat(12, 12, 12, 24, kernel=kernel)
    st = O.starting_state(L, R=True)
    with thirring.Lattice(12, 12, 12, 24, kernel=kernel) as G:
        for dag in (False, True):
            ref = (O.dslashd if dag else O.dslash)(L, st["R"], st["u"], 0.05, imass)
            got = (G.dslashd if dag else G.dslash)(st["R"], st["u"], 0.05, imass)
            assert rel_err(interior(got), interior(ref)) <= TOL


@pytest.mark.gpu
def test_output_halos_are_periodic_images():
    rng = np.random.default_rng(1)
    L = O.lat(4, 4, 4, 8)
    u, R = rand_links(L, rng), rand_spinor(L, rng)
    with thirring.Lattice(4, 4, 4, 8) as G:
        got = G.dslash(R, u, 0.1, 1)
    ref = O.update_halo_5(L, got.copy(order="F"))
    # faces equal their periodic images
    assert np.array_equal(got[0, 1:-1, 1:-1, 1:-1], ref[0, 1:-1, 1:-1, 1:-1])
    assert np.array_equal(got[1:-1, 0, 1:-1, 1:-1], ref[1:-1, 0, 1:-1, 1:-1])
    assert np.array_equal(got[1:-1, 1:-1, 1:-1, -1], ref[1:-1, 1:-1, 1:-1, -1])


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", [0, 1])
def test_even_odd_bit_identical(kernel):
    rng = np.random.default_rng(7)
    L = O.lat(6, 4, 8, 8, kernel=kernel)
    u, R = rand_links(L, rng), rand_spinor(L, rng)
    outs = []
    for layout in (0, 1):
        with thirring.Lattice(6, 4, 8, 8, kernel=kernel, layout=layout) as G:
            outs.append((G.dslash(R, u, 0.02, 3), G.dslashd(R, u, 0.02, 3)))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


@pytest.mark.gpu
def test_wilson_imass5_rejected():
    rng = np.random.default_rng(2)
    L = O.lat(4, 4, 4, 4, kernel=1)
    u, R = rand_links(L, rng), rand_spinor(L, rng)
    with thirring.Lattice(4, 4, 4, 4, kernel=1) as G:
        with pytest.raises(thirring.ThirringError) as ei:
            G.dslash(R, u, 0.1, 5)
        assert ei.value.status == 7


@pytest.mark.gpu
def test_autotuner_keeps_results_bit_identical(tmp_path):
    """The stencil autotuner (register budget per lattice) runs on first use; its
    candidates share block shape and arithmetic, so the output is the same bits
    before and after tuning and equal to a THR_TUNE=0 process."""
    import ctypes as C
    import os
    import subprocess
    import sys
    rng = np.random.default_rng(99)
    L = O.lat(8, 6, 4, 16)
    u = rand_links(L, rng)
    R = rand_spinor(L, rng)
    with thirring.Lattice(8, 6, 4, 16) as G:
        a = G.dslash(R, u, 0.05, 3)
        b = G.dslash(R, u, 0.05, 3)
        buf = C.create_string_buffer(8192)
        thirring.lib().thr_tune_report(buf, len(buf))
    assert np.array_equal(a, b)
    assert "8x6x4 Ls=16" in buf.value.decode()
    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "thirring-rhmc_b200")
    np.save(tmp_path / "R.npy", R)
    np.save(tmp_path / "u.npy", u)
    code = ("import sys, numpy as np; sys.path.insert(0, %r); import thirring; d = %r;"
            "R = np.asfortranarray(np.load(d + '/R.npy')); u = np.asfortranarray(np.load(d + '/u.npy'));"
            "G = thirring.Lattice(8, 6, 4, 16); np.save(d + '/out.npy', G.dslash(R, u, 0.05, 3)); G.close()"
            % (pkg, str(tmp_path)))
    subprocess.run([sys.executable, "-c", code], check=True, env=dict(os.environ, THR_TUNE="0"))
    assert np.array_equal(a, np.load(tmp_path / "out.npy"))


@pytest.mark.gpu
@pytest.mark.parametrize("kernel,force,ls", [(0, "7", 16), (0, "6", 16), (0, "224", 16), (0, "223", 16),
                                             (0, "242", 16), (0, "281", 32), (0, "224", 48), (0, "281", 48),
                                             (0, "108", 16), (0, "106", 32), (1, "3", 16), (1, "2", 16),
                                             (1, "104", 16), (1, "102", 32), (1, "3", 12)])
def test_register_budgets_bit_identical(tmp_path, kernel, force, ls):
    """Every register budget and block shape the stencil tuner may pick gives the
    same bits for M, M^dagger and congrad (whose stencils carry the |Mp|^2 and the
    fused residual-update epilogues): THR_TUNE=<n> forces candidate n (2KM: the
    Shamir blocks of K site groups; 10x: the fifth dimension read from memory
    instead of shuffled, for either kernel), THR_TUNE=0 the default."""
    import os
    import subprocess
    import sys
    rng = np.random.default_rng(7)
    L = O.lat(8, 6, 4, ls)
    u = rand_links(L, rng)
    R = rand_spinor(L, rng)
    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "thirring-rhmc_b200")
    np.save(tmp_path / "R.npy", R)
    np.save(tmp_path / "u.npy", u)
    code = ("import sys, numpy as np; sys.path.insert(0, %r); import thirring; d = %r; t = sys.argv[1];"
            "R = np.asfortranarray(np.load(d + '/R.npy')); u = np.asfortranarray(np.load(d + '/u.npy'));"
            "G = thirring.Lattice(8, 6, 4, %d, kernel=%d); G.set_links(u);"
            "a = G.dslash(R, None, 0.05, 3); b = G.dslashd(R, None, 0.05, 1);"
            "X = np.zeros_like(R); it, _ = G.congrad(R, X, 1e-6, 0.05, 1);"
            "np.savez(d + '/out_' + t + '.npz', a=a, b=b, x=X, it=it); G.close()"
            % (pkg, str(tmp_path), ls, kernel))
    for t in ("0", force):
        subprocess.run([sys.executable, "-c", code, t], check=True, env=dict(os.environ, THR_TUNE=t))
    ref, got = np.load(tmp_path / "out_0.npz"), np.load(tmp_path / ("out_%s.npz" % force))
    for k in ("a", "b", "x", "it"):
        assert np.array_equal(ref[k], got[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("dims,layout", [((8, 6, 4, 16), 0), ((6, 6, 4, 12), 1), ((4, 4, 6, 8), 0)])
def test_split_stencil_bit_identical(tmp_path, dims, layout):
    """The four-threads-per-site FP64 Shamir kernel (autotuner candidate 40, forced by
    THR_TUNE=40) against the one-thread kernel (THR_TUNE=8): the same bits for M and
    M^dagger, every fused epilogue (residual update, h recurrence, with |out|^2), congrad
    and the batched multishift, with the warp-shuffle fifth dimension (Ls 16, 8) and
    without (Ls 12, even-odd order)."""
    import os
    import subprocess
    import sys
    rng = np.random.default_rng(17)
    L = O.lat(*dims)
    np.save(tmp_path / "R.npy", rand_spinor(L, rng))
    np.save(tmp_path / "A.npy", rand_spinor(L, rng))
    np.save(tmp_path / "u.npy", rand_links(L, rng))
    an, ad, _, _ = O.read_remez(os.path.join(os.path.dirname(__file__), "golden", "remez4g"), 12)
    np.save(tmp_path / "an.npy", an)
    np.save(tmp_path / "ad.npy", ad)
    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "thirring-rhmc_b200")
    code = ("import sys, numpy as np; sys.path.insert(0, %r); import thirring; d = %r; t = sys.argv[1];"
            "ld = lambda k: np.asfortranarray(np.load(d + '/' + k + '.npy'));"
            "R, A, u, an, ad = ld('R'), ld('A'), ld('u'), np.load(d + '/an.npy'), np.load(d + '/ad.npy');"
            "G = thirring.Lattice(*%r, layout=%d); G.set_links(u); r = {};"
            "r['a'] = G.dslash(R, None, 0.05, 3); r['b'] = G.dslashd(R, None, 0.05, 1);"
            "r['f1'], r['n1'] = G.dslash_fused(R, A, 0.3, 0.05, 3, True, 1);"
            "r['f3'], r['n3'] = G.dslash_fused(R, A, -0.7, 0.05, 3, False, 3);"
            "X = np.zeros_like(R); r['it'], _ = G.congrad(R, X, 1e-6, 0.05, 1); r['x'] = X;"
            "r['ms'], r['msi'], _ = G.multishift_solver(u, 0.05, 3, ad, an[1:], R, 1e-9, 20000);"
            "np.savez(d + '/out_' + t + '.npz', **r); G.close()" % (pkg, str(tmp_path), dims, layout))
    for t in ("8", "40"):
        subprocess.run([sys.executable, "-c", code, t], check=True, env=dict(os.environ, THR_TUNE=t))
    ref, got = np.load(tmp_path / "out_8.npz"), np.load(tmp_path / "out_40.npz")
    for k in ref.files:
        assert np.array_equal(ref[k], got[k]), k


@pytest.mark.gpu
def test_tiled_stencil_matches_k_dslash(tmp_path):
    """The staged-tile FP64 Shamir kernel (THR_TILE=1) against k_dslash (the
    default, oracle-checked above) in two processes on a lattice both take: M and M^dagger to rounding (the same
    arithmetic, operation for operation), and congrad -- whose stencils carry the
    |Mp|^2 and residual-update epilogues, with partial sums over other blocks --
    to its own tolerance with the iteration count within 1."""
    import os
    import subprocess
    import sys
    rng = np.random.default_rng(71)
    dims = (8, 8, 4, 16)
    L = O.lat(*dims)
    u = rand_links(L, rng)
    R = rand_spinor(L, rng)
    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "thirring-rhmc_b200")
    np.save(tmp_path / "R.npy", R)
    np.save(tmp_path / "u.npy", u)
    code = ("import sys, numpy as np; sys.path.insert(0, %r); import thirring; d = %r; t = sys.argv[1];"
            "R = np.asfortranarray(np.load(d + '/R.npy')); u = np.asfortranarray(np.load(d + '/u.npy'));"
            "G = thirring.Lattice(*%r); G.set_links(u);"
            "a = G.dslash(R, None, 0.05, 3); b = G.dslashd(R, None, 0.05, 1); c = G.dslash(R, None, 0.05, 5);"
            "X = np.zeros_like(R); it, _ = G.congrad(R, X, 1e-8, 0.05, 1);"
            "np.savez(d + '/out_' + t + '.npz', a=a, b=b, c=c, x=X, it=it); G.close()"
            % (pkg, str(tmp_path), dims))
    for t in ("0", "1", "2"):
        subprocess.run([sys.executable, "-c", code, t], check=True, env=dict(os.environ, THR_TILE=t))
    ref, got, got2 = (np.load(tmp_path / ("out_%s.npz" % t)) for t in ("0", "1", "2"))
    for k in ("a", "b", "c"):
        assert rel_err(interior(got[k]), interior(ref[k])) <= 1e-15, k
    assert abs(int(got["it"]) - int(ref["it"])) <= 1
    assert rel_err(interior(got["x"]), interior(ref["x"])) <= 1e-7
    # THR_TILE=2, the persistent double-buffered form: the same tiles, arithmetic and
    # partial-sum order as THR_TILE=1, so the same bits
    for k in ("a", "b", "c", "x", "it"):
        assert np.array_equal(got2[k], got[k]), k


def _dev_dslash(G, R, precision, am, imass, dag):
    import ctypes as C
    L = thirring.lib()
    a, b = C.c_void_p(), C.c_void_p()
    assert L.thr_field_create(G.h, precision, C.byref(a)) == 0
    assert L.thr_field_create(G.h, precision, C.byref(b)) == 0
    try:
        assert L.thr_field_upload(G.h, a, precision, R.ctypes.data_as(C.c_void_p)) == 0
        assert L.thr_dslash_dev(G.h, b, a, precision, am, imass, dag) == 0
        out = np.zeros_like(R)
        assert L.thr_field_download(G.h, out.ctypes.data_as(C.c_void_p), b, precision) == 0
        assert L.thr_sync(G.h) == 0
        return out
    finally:
        L.thr_field_destroy(G.h, a)
        L.thr_field_destroy(G.h, b)


@pytest.mark.gpu
@pytest.mark.parametrize("ls", [5, 6, 8, 48])
@pytest.mark.parametrize("imass", [1, 3, 5])
def test_dslash_fp32_storage(ls, imass):
    """FP32 storage (the single-precision operators of dirac_sp.F90): even Ls runs the
    two-s-per-thread kernel, odd Ls the one-s kernel; both agree with the FP64 oracle
    to single-precision rounding."""
    rng = np.random.default_rng(70 + ls + imass)
    dims = (6, 4, 4, ls)
    L = O.lat(*dims)
    u = rand_links(L, rng)
    R = rand_spinor(L, rng)
    with thirring.Lattice(*dims) as G:
        G.set_links(u)
        for dag in (0, 1):
            got = _dev_dslash(G, R, 1, 0.05, imass, dag)
            ref = (O.dslashd if dag else O.dslash)(L, R, u, 0.05, imass)
            assert rel_err(interior(got), interior(ref)) <= 2e-6, (ls, imass, dag)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["1", "2"])
def test_tile_wait_bound_reports_timeout(tmp_path, mode):
    """The staged-tile stencil's bounded wait.  With THR_TILE_WAIT_TEST=1 every block expects
    16 bytes more than its copies bring, so its wait runs out although every copy has
    completed (nothing faults); each block then writes NaN to all its outputs and counts the
    event (thr_stencil_timeouts).  A normal run of the same kernel counts none."""
    import os
    import subprocess
    import sys
    rng = np.random.default_rng(5)
    dims = (8, 8, 4, 16)  # staged-tile shape: 8*8*4/32 tiles x 16/8 s-chunks = 16 blocks
    L = O.lat(*dims)
    np.save(tmp_path / "R.npy", rand_spinor(L, rng))
    np.save(tmp_path / "u.npy", rand_links(L, rng))
    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "thirring-rhmc_b200")
    code = ("import sys, ctypes as C, numpy as np; sys.path.insert(0, %r); import thirring; d = %r;"
            "R = np.asfortranarray(np.load(d + '/R.npy')); u = np.asfortranarray(np.load(d + '/u.npy'));"
            "G = thirring.Lattice(*%r); G.set_links(u); out = G.dslash(R, None, 0.05, 1);"
            "n = C.c_ulonglong(0); assert thirring.lib().thr_stencil_timeouts(G.h, C.byref(n)) == 0;"
            "np.save(d + '/out_' + sys.argv[1] + '.npy', out); print('timeouts', n.value); G.close()"
            % (pkg, str(tmp_path), dims))
    res = {}
    for tag, env in (("ok", {"THR_TILE": mode}), ("bound", {"THR_TILE": mode, "THR_TILE_WAIT_TEST": "1"})):
        r = subprocess.run([sys.executable, "-c", code, tag], capture_output=True, text=True, timeout=300,
                           env=dict(os.environ, **env))
        assert r.returncode == 0, r.stdout + r.stderr
        res[tag] = int(r.stdout.split("timeouts")[-1].split()[0])
    ok, bound = np.load(tmp_path / "out_ok.npy"), np.load(tmp_path / "out_bound.npy")
    assert res["ok"] == 0 and np.all(np.isfinite(interior(ok)))
    assert res["bound"] == 16 and np.all(np.isnan(interior(bound)))
