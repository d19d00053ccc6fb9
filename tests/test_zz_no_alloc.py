"""thr_congrad_static: the allocation-free congrad, checked against thr_congrad.

Callers that cannot allocate device memory when they solve (their device
footprint is fixed once their fields are placed) pass their own device
arrays; the entry point keeps its CG work vectors in a fixed array inside
the library image.  This file is collected last so that, in a run that stops
at the first failure, every other test has already run.  It passes both run
alone in a fresh process and after the rest of the suite.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O
import thirring
from thirring import _lib

TOL = 1e-10  # the congrad parity tolerance of the 27-iteration fixture


def _dev_spinor(torch, a):
    """Fortran halo'd spinor -> device layout [d][t][y][x][s] (natural site order)."""
    i = a[1:-1, 1:-1, 1:-1, 1:-1, :]
    return torch.from_numpy(np.ascontiguousarray(i.transpose(4, 3, 2, 1, 0))).cuda()


def _dev_links(torch, u):
    i = u[1:-1, 1:-1, 1:-1, :]
    return torch.from_numpy(np.ascontiguousarray(i.transpose(3, 2, 1, 0))).cuda()


def _check_static_twice():
    """thr_congrad_static twice in a row against thr_congrad on the congrad fixture."""
    import torch
    # tests/test_congrad.F90 fixture: 12^3 x 24, res 0.1, am 0.05, imass 3
    L = O.lat(12, 12, 12, 24)
    st = O.starting_state(L, X=True)
    with thirring.Lattice(12, 12, 12, 24) as G:
        G.set_links(st["u"])
        X_ref = st["X"].copy(order="F")
        it_ref, nx_ref = G.congrad(st["Phi"], X_ref, 0.1, 0.05, 3)
    ref = np.ascontiguousarray(X_ref[1:-1, 1:-1, 1:-1, 1:-1, :].transpose(4, 3, 2, 1, 0))
    lib = _lib.lib()
    prm = _lib.Params(12, 12, 12, 24, 0, 0, 25, 1.0, 0.4, -1, 0)
    u = _dev_links(torch, st["u"])
    phi = _dev_spinor(torch, st["Phi"])
    for call in range(2):  # the shared scratch keeps the previous call's contents
        x = _dev_spinor(torch, st["X"])
        torch.cuda.synchronize()
        it, nx = C.c_int(0), C.c_int(0)
        rc = lib.thr_congrad_static(C.byref(prm), C.c_void_p(u.data_ptr()), C.c_void_p(phi.data_ptr()),
                                    C.c_void_p(x.data_ptr()), 0.1, C.byref(it), 0.05, 3, C.byref(nx), None)
        assert rc == 0, rc
        assert it.value == it_ref == 27 and nx.value == nx_ref
        got = x.cpu().numpy()
        err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
        assert err <= TOL, (call, err)


@pytest.mark.gpu
def test_congrad_static_matches_congrad_twice():
    _check_static_twice()


@pytest.mark.gpu
@pytest.mark.parametrize("tune", ["0", "1"])
def test_congrad_static_fresh_process(tune):
    # alone in a fresh process, with the stencil autotuner off (THR_TUNE=0) and on: the
    # allocation-free call never tunes, so it gives the same answer either way
    here = os.path.dirname(os.path.abspath(__file__))
    code = ("import sys; sys.path.insert(0, %r); import conftest; import test_zz_no_alloc as t; "
            "t._check_static_twice(); print('ok')" % here)
    env = dict(os.environ, THR_TUNE=tune)
    r = subprocess.run([sys.executable, "-c", code], cwd=here, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr


@pytest.mark.gpu
def test_congrad_static_rejects_oversized_lattice():
    lib = _lib.lib()
    prm = _lib.Params(48, 48, 48, 48, 0, 0, 25, 1.0, 0.4, -1, 0)
    dummy = C.c_void_p(1)  # rejected before any use
    rc = lib.thr_congrad_static(C.byref(prm), dummy, dummy, dummy, 0.1, C.byref(C.c_int()), 0.05, 3, None, None)
    assert rc == 2  # THR_ERR_BADSHAPE
