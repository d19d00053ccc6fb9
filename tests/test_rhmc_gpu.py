"""RHMC layer on the GPU vs the oracle: force, hamilton, initialise_phi /
initialise_pp, and whole trajectories (force_module.F90, dwf3d_lib.F90,
evolution.F90), with the reference's own remez coefficient files.

Bounds: FP64 guidance solves give forces within 1e-9 and Delta H within
1e-6 (absolute) of the FP64 oracle; the single-precision guidance solver
(spmd, multishift_solver_sp) within 1e-4 on the force and SPMD_DH_BOUND on
Delta H against the oracle's own single-precision trajectory.
"""
import os

import numpy as np
import pytest

import oracle as O
import thirring
from helpers import interior, rand_theta, rel_err

GOLD = os.path.join(os.path.dirname(__file__), "golden")

# The reference's single-precision guidance solves (spmd = 1) change the trajectory
# itself: in the oracle alone, Delta H of these 3-step trajectories moves by up to 2.2e-5
# against FP64 guidance (seeds 9, 11, 13).  GPU and oracle, both in single precision,
# round their FP32 sums in different orders and differ by up to 1.6e-5 on the same
# trajectories (measured on B200); FP64 guidance agrees to 6e-8, within the 1e-6 bar.
SPMD_DH_BOUND = 5e-5


def rats():
    g = os.path.join(GOLD, "")
    rat = thirring.remez_set(g + "remez2", g + "remez4", 25)
    ratg = thirring.remez_set(g + "remez2g", g + "remez4g", 12)
    return rat, ratg


def setup(kernel=0, dims=(4, 4, 4, 8), beta=0.4, seed=5):
    rng = np.random.default_rng(seed)
    L = O.lat(*dims, kernel=kernel, beta=beta)
    theta = rand_theta(L, rng, beta)
    rat, ratg = rats()
    G = thirring.Lattice(*dims, kernel=kernel, beta=beta)
    G.set_remez(rat, ratg)
    return L, G, theta, O.rational(rat, ratg), rng


@pytest.mark.gpu
@pytest.mark.parametrize("kernel,spmd", [(0, 0), (0, 1), (1, 0)])
def test_force(kernel, spmd):
    L, G, theta, orat, rng = setup(kernel)
    from helpers import rand_spinor
    Phi = rand_spinor(L, rng)
    u = O.coef(L, theta)
    ref = O.force(L, u, theta, orat, Phi, 1e-8 if not spmd else 1e-6, 0.05, 3, spmd)
    with G:
        G.coef(theta)
        G.set_residuals(spmd=spmd)
        got = G.force(Phi, 1e-8 if not spmd else 1e-6, 0.05, 3, theta)
    assert rel_err(got, ref) <= (1e-9 if not spmd else 1e-4)


@pytest.mark.gpu
def test_hamilton():
    L, G, theta, orat, rng = setup()
    from helpers import rand_spinor
    Phi = rand_spinor(L, rng)
    pp = np.asfortranarray(rng.standard_normal((4, 4, 4, 3)), np.float32)
    u = O.coef(L, theta)
    ref = O.hamilton(L, u, theta, pp, orat, Phi, 1e-8, 0.05, 3)
    with G:
        G.coef(theta)
        got = G.hamilton(Phi, 1e-8, 0.05, 3, theta, pp)
    for a, b in zip(got, ref):
        assert abs(a - b) <= 1e-10 * abs(b)


@pytest.mark.gpu
def test_initialise_phi_pp():
    L, G, theta, orat, rng = setup()
    g = O.RNG(L, True).init(4139764973254.0)
    u = O.coef(L, theta)
    ref_phi = O.initialise_phi(L, g, u, orat, 0.05, 3)
    ref_pp = O.initialise_pp(L, g)
    with G:
        G.coef(theta)
        G.init_random(4139764973254.0, site=True)
        phi = G.initialise_phi(0.05, 3)
        pp = G.initialise_pp()
    assert rel_err(interior(phi), interior(ref_phi)) <= 1e-8
    assert np.max(np.abs(pp - ref_pp)) <= 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("spmd", [0, 1])
def test_trajectory_delta_h(spmd):
    # fixed-length trajectories (3 steps, dt = 0.05) from the same theta and seed
    L, G, theta, orat, rng = setup(beta=0.4, seed=9)
    g = O.RNG(L, True).init(4139764973254.0)
    th_ref = theta.copy(order="F")
    refs = [O.trajectory(L, g, th_ref, orat, 3, 0.05, 0.05, 3, 1e-8, 1e-6, spmd, fixed_steps=3) for _ in range(2)]
    with G:
        G.init_random(4139764973254.0, site=True)
        G.set_residuals(1e-8, 1e-6, spmd)
        th = theta.copy(order="F")
        gots = [G.trajectory(th, 3, 0.05, 0.05, 3, fixed_steps=3) for _ in range(2)]
    for got, ref in zip(gots, refs):
        assert got.steps == ref.steps == 3
        assert abs(got.dh - ref.dh) <= (1e-6 if spmd == 0 else SPMD_DH_BOUND), (got.dh, ref.dh)
        assert got.accepted == ref.accepted
    assert np.max(np.abs(th - th_ref)) <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("spmd", [0, 1])
def test_trajectory_mixed_action_delta_h(spmd):
    """The Hamiltonian and pseudofermion solves in the mixed multishift (FP64 until the
    residual is small, then FP32 with FP64 shift fields): Delta H within 1e-6 of the
    FP64 oracle's with FP64 guidance, as the FP64 path."""
    L, G, theta, orat, rng = setup(beta=0.4, seed=9)
    g = O.RNG(L, True).init(4139764973254.0)
    th_ref = theta.copy(order="F")
    ref = O.trajectory(L, g, th_ref, orat, 3, 0.05, 0.05, 3, 1e-8, 1e-6, spmd, fixed_steps=3)
    with G:
        G.init_random(4139764973254.0, site=True)
        G.set_residuals(1e-8, 1e-6, spmd)
        G.set_action_precision(thirring.MIXED_FP32)
        G.set_mixed(1e-6, 1e-13)  # early enough that this small solve switches
        th = theta.copy(order="F")
        got = G.trajectory(th, 3, 0.05, 0.05, 3, fixed_steps=3)
    assert got.steps == ref.steps == 3
    assert abs(got.dh - ref.dh) <= (1e-6 if spmd == 0 else SPMD_DH_BOUND), (got.dh, ref.dh)


def _traj_run(tmp, tag):
    """Two fixed-length and two random-length trajectories; results saved for comparison."""
    import sys
    L, G, theta, orat, rng = setup(beta=0.4, seed=13)
    out = {}
    with G:
        G.init_random(4139764973254.0, site=True)
        G.set_residuals(1e-8, 1e-6, 1)
        th = theta.copy(order="F")
        rs = [G.trajectory(th, 4, 0.05, 0.05, 3, fixed_steps=4) for _ in range(2)]
        rs += [G.trajectory(th, 3, 0.05, 0.05, 3) for _ in range(2)]
        out["dh"] = np.array([r.dh for r in rs])
        out["steps"] = np.array([r.steps for r in rs])
        out["acc"] = np.array([r.accepted for r in rs])
        out["theta"] = th
        out["counts"] = np.array(list(G.md_counters().values()))
    np.savez(os.path.join(tmp, "traj_%s.npz" % tag), **out)


@pytest.mark.gpu
def test_md_step_graph_bit_identical(tmp_path):
    """A leapfrog step replayed as one captured CUDA graph (drift, coef, the four force
    solves with their batch loops as conditional nodes, the exit draw, the kick) runs
    exactly the kernels of the host-driven step: identical Delta H, steps, theta and
    iteration counts for fixed and random trajectory lengths (THR_MD_GRAPH=0: host-driven)."""
    import subprocess
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    code = ("import sys; sys.path.insert(0, %r); import conftest; import test_rhmc_gpu as t; t._traj_run(%r, sys.argv[1])"
            % (here, str(tmp_path)))
    for tag, env in (("graph", {}), ("host", {"THR_MD_GRAPH": "0"})):
        subprocess.run([sys.executable, "-c", code, tag], check=True, cwd=here, env=dict(os.environ, **env))
    a, b = np.load(tmp_path / "traj_graph.npz"), np.load(tmp_path / "traj_host.npz")
    assert list(a["steps"][:2]) == [4, 4]  # the fixed-length pair replays the step graph three times each
    for k in a.files:
        assert np.array_equal(a[k], b[k]), k
