#!/usr/bin/env python
"""Headline benchmark: the rational-approximation multishift solve (qmrherm).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--mode fp64|mixed]

Workload (one "step"): qmrherm iflag 0 -- x = sum_i a_i (M^dagger M + s_i)^-1 Phi --
on a 32^2 x 32 lattice with Ls = 32 (Shamir kernel, am = 0.01, imass = 1,
domain-wall height 1), 25 poles s_i log-spaced in [1e-5, 1e2] with positive
residues of the x^-1/2 form, solved to the reference's residual 1e-9.
theta is Gaussian with variance 1/beta (beta = 0.3) and Phi is a complex
Gaussian source, both seeded (synthetic: the reference publishes no data
set).  The working set (2 x 25 shift fields of 67 MB) is far larger than L2,
so no flush is needed between steps.

Reported: `value` = solves/s over all ranks with inputs resident in HBM;
`e2e` = the same through the C-ABI call with host Fortran-layout arrays
(pinned), host<->device copies inside the timed region; `roofline` for the
dominant kernel, timed live with CUDA events on the library's stream;
`cpu_baseline` = the oracle (C restatement of the reference) on this host's
cores over a bounded sample of the same solve.  With N > 1 (torchrun), each
rank solves its own replica lattice (no collective on the data path) and the
timing is the max over ranks.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "thirring-rhmc_b200"))

# ------------------------------------------------------------------ workload
LX = LY = LT = 32
LS = 32
BETA, AM, IMASS, AM3, RES = 0.3, 0.01, 1, 1.0, 1e-9
NPOLE = 25
# iterations the FP64 multishift takes on this seeded input (used to scale
# the CPU sample to whole solves; re-measured by every GPU run and printed)
FP64_ITERS_REF = 17113  # measured on B200 for the seeded input below
METRIC = "multishift solve throughput (qmrherm, 25 poles, FP64 residual 1e-9)"
# kernel timing inside the timed region: every PROF_STRIDE-th launch of each kind
PROF_STRIDE = 8
PROF_KINDS = ((0, "k_dslash_M_hrec"), (2, "k_dslash_Mdag"), (1, "k_flush"), (3, "k_dslash_M_hrec_fp32"),
              (4, "k_dslash_Mdag_fp32"), (5, "k_alpha"), (6, "k_lambda"))
UNIT = "solves/s"
HBM_FALLBACK = 6650.0
# arithmetic of each mode: the mixed modes run FP64 first and FP32 (BF16 storage,
# FP32 arithmetic) once the residual is small, with FP64 shift fields throughout
DTYPES = {"fp64": "f64", "sp": "f32", "mixed": "f64+f32", "bf16": "f64+bf16"}


def rational():
    s = np.logspace(-5.0, 2.0, NPOLE)
    delta = 7.0 / (NPOLE - 1)  # decades between poles
    a = np.sqrt(s) * delta * np.log(10.0) / np.pi  # x^-1/2 ~ (1/pi) int ds s^-1/2/(s+x)
    return np.concatenate([[0.0], a]), s


def inputs(rank):
    rng = np.random.default_rng(20240 + rank)
    theta = np.asfortranarray(rng.standard_normal((LX, LY, LT, 3)) / np.sqrt(BETA), np.float32)
    phi = np.zeros((LS + 2, LX + 2, LY + 2, LT + 2, 4), np.complex128, order="F")
    shp = phi[1:-1, 1:-1, 1:-1, 1:-1, :].shape
    phi[1:-1, 1:-1, 1:-1, 1:-1, :] = rng.standard_normal(shp) + 1j * rng.standard_normal(shp)
    return theta, phi


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK, "fallback"


def ncu_traffic(kernel, algorithmic_per_launch):
    """per-launch DRAM bytes of `kernel` from the committed ncu summary: a measured
    figure ("traffic <kernel> <bytes>") or a measured traffic/algorithmic ratio applied
    to this launch ("ratio <kernel> <r>"); None if neither was recorded"""
    p = os.path.join(REPO, "profiles", "roofline_traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        f = line.split()
        if len(f) >= 3 and f[1] == kernel:
            if f[0] == "traffic":
                return float(f[2])
            if f[0] == "ratio":
                return round(float(f[2]) * algorithmic_per_launch)
    return None


class Clocks:
    """nvidia-smi sampling during the timed region"""

    def __init__(self, dev):
        self.dev = dev
        self.p = None
        self.out = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.p = None
        return self

    def _read(self):
        for line in self.p.stdout:
            self.out.append(line.strip())

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ replicas
def max_over_ranks(x, world):
    """The slowest rank's time: one all-reduce(MAX) of a float64 scalar on the
    process group's device (CUDA under NCCL, CPU under gloo)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, steps, ms_max):
    """Whole-job solves/s: every rank solves its own replica lattice `steps`
    times; the job takes as long as its slowest rank."""
    return world * steps / (ms_max / 1e3)


# ------------------------------------------------------------------ GPU arm
def run_ours(args, rank, world, local_rank):
    import torch
    import thirring
    from thirring import _lib

    torch.cuda.set_device(local_rank)
    L = _lib.lib()
    mode = {"fp64": 0, "sp": 1, "mixed": 2, "bf16": 3}[args.mode]
    anum, aden = rational()
    theta, phi = inputs(rank)
    G = thirring.Lattice(LX, LY, LT, LS, kernel=0, beta=BETA, am3=AM3, device=local_rank)
    G.coef(theta)
    h = G.h
    pd = C.c_void_p()
    px = C.c_void_p()
    assert L.thr_field_create(h, 0, C.byref(pd)) == 0 and L.thr_field_create(h, 0, C.byref(px)) == 0
    assert L.thr_field_upload(h, pd, 0, phi.ctypes.data_as(C.c_void_p)) == 0
    an = np.ascontiguousarray(anum)
    ad = np.ascontiguousarray(aden)
    it = C.c_int(0)
    cgr = np.zeros(NPOLE, np.int32)

    if args.max_iters:
        L.thr_set_residuals(h, 1e-8, 1e-6, 1, args.max_iters)

    def solve(m):
        rc = L.thr_qmrherm_dev(h, pd, px, RES, C.byref(it), AM, IMASS, an.ctypes.data_as(C.c_void_p),
                               ad.ctypes.data_as(C.c_void_p), NPOLE, 0, m, cgr.ctypes.data_as(C.c_void_p))
        if rc != 0 and not (args.max_iters and rc == 3):  # 3: THR_ERR_MAXITER, expected when capped
            raise RuntimeError(f"thr_qmrherm_dev failed: {rc}")
        return it.value

    sptr = C.c_void_p()
    L.thr_get_stream(h, C.byref(sptr))
    stream = torch.cuda.ExternalStream(sptr.value)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def tmax(x):
        return max_over_ranks(x, world)

    # ---- warm-up
    iters = 0
    for _ in range(args.warmup):
        iters = solve(mode)
    # ---- timed region (inputs resident), profiled kernels, sampled clocks
    # The solves run as one CUDA graph each; the last timed step is launched from
    # the host with every PROF_STRIDE-th launch of each profiled kernel bracketed
    # by events (same kernels; its launch gaps count against the timed value).
    L.thr_profile(h, 0, 1)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    its = []
    with Clocks(local_rank) as clk:
        e0.record(stream)
        for i in range(args.steps):
            if i == args.steps - 1:
                L.thr_profile(h, PROF_STRIDE, 0)
            its.append(solve(mode))
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = tmax(e0.elapsed_time(e1))
    L.thr_profile(h, 0, 0)
    prof = {}
    for kind, name in PROF_KINDS:
        n = C.c_int(0)
        t = C.c_double(0)
        b = C.c_double(0)
        tot = C.c_double(0)
        L.thr_profile_read(h, kind, C.byref(n), C.byref(t), C.byref(b), C.byref(tot))
        prof[name] = dict(sampled=n.value, ms=t.value, bytes=b.value, launches=tot.value)
    # ---- accuracy of the timed solves: the true residual of every shifted system of
    # the last one (FP64, on the device), against the stopping rule of
    # multishift_module.F90:244 (|r_k| * correction_k < res)
    acc = shift_accuracy(L, h, pd, ad, an)
    acc["left_fp64_at_iteration"] = G.mixed_switched_at() if mode in (2, 3) else None
    # the batched FP64 solve (the arm mode would replace) timed once for the ratio, and
    # for a low-precision mode the per-shift error of its solutions against it
    fp64b_s = None
    if mode != 0:
        torch.cuda.synchronize()
        e0.record(stream)
        it64 = solve(0)
        e1.record(stream)
        e1.synchronize()
        fp64b_s = e0.elapsed_time(e1) / 1e3
        acc["fp64_iterations"] = it64
        acc["fp64_shift_true_residual"] = shift_accuracy(L, h, pd, ad, an)
        acc["per_shift_rel_error_vs_fp64"] = shift_errors_vs_fp64(G, phi, anum, aden, mode)
    # the batched solver's graph runs batches in pairs: a batch is 32 iterations of 4
    # kernels (M with the h recurrence and |h|^2, alpha, M^dagger with the residual
    # update, lambda) plus the previous batch's flush (coefficients, flush, history
    # reset), a pair ends in the loop control; per solve 3 set-up kernels, the last
    # batch's flush and the pole sum
    def batch_launches(i):
        pairs = (i + 63) // 64
        return 3 + pairs * (2 * (32 * 4 + 3) + 1) + 3 + 1
    launches = int(sum(batch_launches(i) for i in its))

    # ---- plain FP64 GPU path for comparison: FP64 everywhere and the reference's
    # loop structure (every shift field updated in every iteration)
    fp64_s, fp64_iters = None, None
    if args.compare_plain:
        L.thr_set_solver(h, 0)
        torch.cuda.synchronize()
        e0.record(stream)
        fp64_iters = solve(0)
        e1.record(stream)
        e1.synchronize()
        fp64_s = e0.elapsed_time(e1) / 1e3
        L.thr_set_solver(h, 1)

    # ---- the same batched solver launched batch by batch from the host (no graph)
    stream_s = None
    if args.compare_plain:
        L.thr_set_solver(h, 2)
        torch.cuda.synchronize()
        e0.record(stream)
        solve(mode)
        e1.record(stream)
        e1.synchronize()
        stream_s = e0.elapsed_time(e1) / 1e3
        L.thr_set_solver(h, 1)

    # ---- e2e through the host C ABI (pinned Fortran-layout arrays)
    x = np.zeros_like(phi)
    for a in (phi, x):
        L.thr_host_register(a.ctypes.data_as(C.c_void_p), a.nbytes)
    e2e_ms = None
    if args.e2e_steps > 0:
        G.qmrherm(phi, RES, AM, IMASS, anum, aden, 0, use_sp=mode)
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.e2e_steps):
            rc = L.thr_qmrherm(h, phi.ctypes.data_as(C.c_void_p), x.ctypes.data_as(C.c_void_p), RES, C.byref(it), AM,
                               IMASS, an.ctypes.data_as(C.c_void_p), ad.ctypes.data_as(C.c_void_p), NPOLE, 0, mode,
                               None, None, None, 0)
            assert rc == 0, rc
        e1.record(stream)
        e1.synchronize()
        barrier()
        e2e_ms = tmax(e0.elapsed_time(e1))
    for a in (phi, x):
        L.thr_host_unregister(a.ctypes.data_as(C.c_void_p))

    # ---- stencil bandwidth at the largest config-2 lattice (extra figure)
    dslash = dslash_bandwidth(args, local_rank) if (rank == 0 and not args.no_dslash) else None

    buf = C.create_string_buffer(8192)
    L.thr_tune_report(buf, len(buf))
    tune = [ln for ln in buf.value.decode().splitlines() if ln]
    res = dict(ms=ms, its=its, prof=prof, launches=launches, fp64_s=fp64_s, fp64_iters=fp64_iters, stream_s=stream_s,
               tune=tune, accuracy=acc, fp64_batched_s=fp64b_s,
               e2e_ms=e2e_ms, clocks=clk.summary(), dslash=dslash, phi_bytes=phi.nbytes)
    L.thr_field_destroy(h, pd)
    L.thr_field_destroy(h, px)
    G.close()
    return res


def correction(anum, aden):
    """multishift_module.F90:87-88: |anum/aden| over its geometric mean"""
    c = np.abs(np.asarray(anum[1:]) / np.asarray(aden))
    return c / np.exp(np.mean(np.log(c)))


def shift_accuracy(L, h, pd, ad, an):
    """True residual |Phi - (M^dagger M + aden_k) x_k| of every shifted solution of the
    context's last solve (thr_shift_residuals_dev), times correction_k, over res."""
    r2 = np.zeros(len(ad))
    rc = L.thr_shift_residuals_dev(h, pd, None, len(ad), ad.ctypes.data_as(C.c_void_p), AM, IMASS,
                                   r2.ctypes.data_as(C.c_void_p))
    if rc != 0:
        return {"error": rc}
    t = np.sqrt(r2) * correction(an, ad) / RES
    return {"max_true_residual_over_res": float(t.max()), "shift_of_max": int(t.argmax()),
            "per_shift_true_residual_over_res": [float("%.3g" % v) for v in t],
            "rule": "|Phi - (M^dagger M + aden_k) x_k| * correction_k / res (multishift_module.F90:244 tests the "
                    "recursive residual against 1)"}


def shift_errors_vs_fp64(G, phi, anum, aden, mode):
    """|x_k - x_k(FP64)| / |x_k(FP64)| per shift, both solves through the C ABI (iflag 1
    returns the shifted solutions in Phi0)."""
    outs = []
    for m in (0, mode):
        Phi0 = np.zeros(G.sshape + (G.ndiag,), np.complex128, order="F")
        G.qmrherm(phi, RES, AM, IMASS, anum, aden, 1, use_sp=m, Phi0=Phi0)
        outs.append(Phi0)
    err = []
    for k in range(len(aden)):
        a = outs[1][1:-1, 1:-1, 1:-1, 1:-1, :, k]
        b = outs[0][1:-1, 1:-1, 1:-1, 1:-1, :, k]
        err.append(float("%.3g" % (np.linalg.norm(a - b) / np.linalg.norm(b))))
    return err


def run_overlap(args):
    """The overlap operator of measure_OWilson.F90: odslash / odslashd at 48^2x48,
    Ls = 16 (algorithmic GB/s: one read of the input spinor, one write of the
    output, three link fields; 0.23 GB per launch, above L2) and congradO on
    16^2x16, Ls = 8 with the reference's prepZolo coefficients (0.1, 5)."""
    import torch
    import thirring
    from thirring import _lib
    L = _lib.lib()
    out = {}
    lx, ls = 48, 16
    G = thirring.Lattice(lx, lx, lx, ls, kernel=1)
    rng = np.random.default_rng(7)
    G.coef(np.asfortranarray(rng.standard_normal((lx, lx, lx, 3)) / np.sqrt(BETA), np.float32))
    a, b = C.c_void_p(), C.c_void_p()
    L.thr_field_create(G.h, 0, C.byref(a))
    L.thr_field_create(G.h, 0, C.byref(b))
    R = thirring.spinor(G)
    R[1:-1, 1:-1, 1:-1, 1:-1, :] = rng.standard_normal(R[1:-1, 1:-1, 1:-1, 1:-1, :].shape)
    L.thr_field_upload(G.h, a, 0, R.ctypes.data_as(C.c_void_p))
    s = C.c_void_p()
    L.thr_get_stream(G.h, C.byref(s))
    st = torch.cuda.ExternalStream(s.value)
    v3 = lx ** 3
    byts = 2 * 4 * ls * v3 * 16 + 3 * v3 * 16
    for dag in (0, 1):
        for _ in range(max(args.warmup, 3)):
            L.thr_odslash_dev(G.h, b, a, AM, 1, dag)
        L.thr_sync(G.h)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            L.thr_odslash_dev(G.h, b, a, AM, 1, dag)
        e1.record(st)
        e1.synchronize()
        us = e0.elapsed_time(e1) / args.steps * 1e3
        out["odslashd" if dag else "odslash"] = {"us": round(us, 2), "gbs": round(byts / us / 1e3, 1)}
    L.thr_field_destroy(G.h, a)
    L.thr_field_destroy(G.h, b)
    G.close()
    lx, ls = 16, 8
    G = thirring.Lattice(lx, lx, lx, ls, kernel=1)
    G.coef(np.asfortranarray(rng.standard_normal((lx, lx, lx, 3)) / np.sqrt(BETA), np.float32))
    Phi = thirring.spinor(G)
    Phi[1:-1, 1:-1, 1:-1, 1:-1, :] = rng.standard_normal(Phi[1:-1, 1:-1, 1:-1, 1:-1, :].shape)
    G.congrad_o(Phi, 1e-6, AM, 1)  # warm-up
    t0 = time.perf_counter()
    X, it, nx = G.congrad_o(Phi, 1e-6, AM, 1)
    dt = time.perf_counter() - t0
    out["congrad_o_16x16x16_ls8"] = {"s": round(dt, 4), "itercg": it, "us_per_iteration": round(dt / max(it, 1) * 1e6, 2),
                                     "res": 1e-6, "am": AM, "zolo": [0.1, 5.0]}
    G.close()
    return {"workload": "overlap operator (measure_OWilson.F90): odslash/odslashd 48^2x48 Ls16, congradO 16^3 Ls8",
            "results": out}


def run_dslash_sweep(args):
    """The config-2 sweep: M and M^dagger at L^2 x L for L in {16, 24, 32, 48} and Ls in
    {16, 32, 48}, FP64 and FP32 storage, Shamir and Wilson kernels, natural and even-odd
    site order.  Per case: the mean of `steps` launches (after `warmup`) timed with CUDA
    events on the library's stream, algorithmic GB/s (one read of the input spinor, one
    write of the output, three link fields) and its fraction of the measured HBM copy
    rate, and the largest deviation from the oracle's FP64 operator (dirac.F90) relative
    to its largest element (natural order; the even-odd order gives the same bits)."""
    import torch
    import thirring
    from thirring import _lib
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    L = _lib.lib()
    peak, peak_kind = peaks()
    sizes = [int(v) for v in (args.sweep_l or "16,24,32,48").split(",")]
    lss = [int(v) for v in (args.sweep_ls or "16,32,48").split(",")]
    steps, warmup = max(args.steps, 5), max(args.warmup, 3)
    cases = []
    for lx in sizes:
        for ls in lss:
            rng = np.random.default_rng(1000 * lx + ls)
            theta = np.asfortranarray(rng.standard_normal((lx, lx, lx, 3)) / np.sqrt(BETA), np.float32)
            R = np.zeros((ls + 2, lx + 2, lx + 2, lx + 2, 4), np.complex128, order="F")
            sh = R[1:-1, 1:-1, 1:-1, 1:-1, :].shape
            R[1:-1, 1:-1, 1:-1, 1:-1, :] = rng.standard_normal(sh) + 1j * rng.standard_normal(sh)
            v3 = lx ** 3
            for kernel, kname in ((0, "shamir"), (1, "wilson")):
                Lo = O.lat(lx, lx, lx, ls, kernel=kernel, beta=BETA, am3=AM3)
                u = O.coef(Lo, theta)
                O.update_halo_5(Lo, R)
                refs = {dag: (O.dslashd if dag else O.dslash)(Lo, R, u, AM, IMASS) for dag in (0, 1)}
                scale = {dag: float(np.max(np.abs(O.interior(refs[dag])))) for dag in (0, 1)}
                for layout, lname in ((0, "natural"), (1, "even_odd")):
                    G = thirring.Lattice(lx, lx, lx, ls, kernel=kernel, layout=layout, beta=BETA, am3=AM3)
                    G.set_links(u)
                    sptr = C.c_void_p()
                    L.thr_get_stream(G.h, C.byref(sptr))
                    st = torch.cuda.ExternalStream(sptr.value)
                    for prec, pname, b in ((0, "fp64", 16), (2, "fp32", 8)):
                        a, o = G._field(prec, R), G._field(prec)
                        for dag in (0, 1):
                            for _ in range(warmup):
                                L.thr_dslash_dev(G.h, o, a, prec, AM, IMASS, dag)
                            L.thr_sync(G.h)
                            e0 = torch.cuda.Event(enable_timing=True)
                            e1 = torch.cuda.Event(enable_timing=True)
                            e0.record(st)
                            for _ in range(steps):
                                L.thr_dslash_dev(G.h, o, a, prec, AM, IMASS, dag)
                            e1.record(st)
                            e1.synchronize()
                            us = e0.elapsed_time(e1) / steps * 1e3
                            byts = 2 * 4 * ls * v3 * b + 3 * v3 * b
                            case = {"L": lx, "Ls": ls, "kernel": kname, "layout": lname, "storage": pname,
                                    "op": "Mdag" if dag else "M", "us": round(us, 2),
                                    "gbs": round(byts / us / 1e3, 1), "frac": round(byts / us / 1e3 / peak, 3)}
                            if layout == 0:
                                out = thirring.spinor(G)
                                L.thr_field_download(G.h, out.ctypes.data_as(C.c_void_p), o, prec)
                                dev = np.max(np.abs(O.interior(out) - O.interior(refs[dag])))
                                case["max_rel_dev_vs_oracle"] = float("%.3g" % (dev / scale[dag]))
                            cases.append(case)
                            print(json.dumps(case), flush=True)
                        L.thr_field_destroy(G.h, a)
                        L.thr_field_destroy(G.h, o)
                    G.close()
    best = max(cases, key=lambda c: c["frac"])
    return {"workload": "config-2 dslash sweep: M and M^dagger, L^2xL L in %s, Ls in %s, FP64/FP32, Shamir/Wilson, "
                        "natural/even-odd, am=%g imass=%d beta=%g" % (sizes, lss, AM, IMASS, BETA),
            "peak_gbs": peak, "peak_source": peak_kind, "launches_per_case": steps, "cases": cases,
            "best": best}


def run_aux_kernels(args):
    """The other bandwidth-bound kernels of the path on the headline lattice (or --lx/--ls):
    derivs (derivs_module.F90:99-196; reads R and X2 once, reads and writes dSdpi) for
    iflag 0 and 1, and the pseudofermion draw of initialise_phi_1flavour (evolution.F90:
    40-51; 4 Ls Gaussian pairs per site: reads and writes each site's generator state, 97
    table entries and 16 bytes, writes the FP64 field).  Per kernel: the mean of `steps`
    launches after `warmup`, CUDA events on the library's stream, algorithmic GB/s and the
    fraction of the measured HBM copy rate."""
    import torch
    import thirring
    from thirring import _lib
    L = _lib.lib()
    peak, peak_kind = peaks()
    lx, ls = LX, LS
    G = thirring.Lattice(lx, lx, lx, ls, beta=BETA)
    rng = np.random.default_rng(11)
    G.coef(np.asfortranarray(rng.standard_normal((lx, lx, lx, 3)) / np.sqrt(BETA), np.float32))
    G.init_random(4139764973254.0)
    R = thirring.spinor(G)
    sh = R[1:-1, 1:-1, 1:-1, 1:-1, :].shape
    R[1:-1, 1:-1, 1:-1, 1:-1, :] = rng.standard_normal(sh) + 1j * rng.standard_normal(sh)
    a, b = G._field(0, R), G._field(0, R)
    sptr = C.c_void_p()
    L.thr_get_stream(G.h, C.byref(sptr))
    st = torch.cuda.ExternalStream(sptr.value)
    v3, n = lx ** 3, 4 * ls * lx ** 3
    steps, warmup = max(args.steps, 10), max(args.warmup, 3)
    out = {}

    def timed(name, fn, byts):
        for _ in range(warmup):
            fn()
        L.thr_sync(G.h)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            fn()
        e1.record(st)
        e1.synchronize()
        us = e0.elapsed_time(e1) / steps * 1e3
        out[name] = {"us": round(us, 2), "algorithmic_bytes": int(byts), "gbs": round(byts / us / 1e3, 1),
                     "frac": round(byts / us / 1e3 / peak, 3)}

    for iflag in (0, 1):
        timed("k_derivs_iflag%d" % iflag, lambda: L.thr_derivs_dev(G.h, a, b, 0.37, iflag, AM, IMASS),
              2 * n * 16 + 2 * 3 * v3 * 8)
    timed("k_phi_draw", lambda: L.thr_phi_draw_dev(G.h, a), n * 16 + 2 * v3 * (97 * 4 + 16))
    L.thr_field_destroy(G.h, a)
    L.thr_field_destroy(G.h, b)
    G.close()
    return {"workload": "auxiliary kernels at %d^2x%d, Ls=%d: derivs (iflag 0, 1), pseudofermion draw" % (lx, lx, ls),
            "peak_gbs": peak, "peak_source": peak_kind, "launches": steps, "results": out}


def dslash_bandwidth(args, dev, lx=48, ls=48, iters=20, warmup=3):
    """FP64 Shamir M at lx^2 x lx, Ls = ls: algorithmic GB/s over `iters` launches
    (one read of the input spinor, one write of the output, three link fields)."""
    import torch
    import thirring
    from thirring import _lib
    L = _lib.lib()
    G = thirring.Lattice(lx, lx, lx, ls, device=dev)
    rng = np.random.default_rng(7)
    G.coef(np.asfortranarray(rng.standard_normal((lx, lx, lx, 3)) / np.sqrt(BETA), np.float32))
    a, b = C.c_void_p(), C.c_void_p()
    L.thr_field_create(G.h, 0, C.byref(a))
    L.thr_field_create(G.h, 0, C.byref(b))
    R = thirring.spinor(G)
    R[1:-1, 1:-1, 1:-1, 1:-1, :] = rng.standard_normal(R[1:-1, 1:-1, 1:-1, 1:-1, :].shape)
    L.thr_field_upload(G.h, a, 0, R.ctypes.data_as(C.c_void_p))
    s = C.c_void_p()
    L.thr_get_stream(G.h, C.byref(s))
    st = torch.cuda.ExternalStream(s.value)
    out = {}
    for dag in (0, 1):
        for _ in range(warmup):
            L.thr_dslash_dev(G.h, b, a, 0, AM, IMASS, dag)
        L.thr_sync(G.h)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(iters):
            L.thr_dslash_dev(G.h, b, a, 0, AM, IMASS, dag)
        e1.record(st)
        e1.synchronize()
        us = e0.elapsed_time(e1) / iters * 1e3
        v3 = lx ** 3
        byts = 2 * 4 * ls * v3 * 16 + 3 * v3 * 16
        out["dslashd" if dag else "dslash"] = {"us": round(us, 2), "gbs": round(byts / us / 1e3, 1)}
    L.thr_field_destroy(G.h, a)
    L.thr_field_destroy(G.h, b)
    G.close()
    return out


# ------------------------------------------------------------------ CPU arm
def cpu_sample(iters_sample, threads=None):
    """Seconds per multishift iteration of the oracle on this workload: FP64
    multishift_solver restated in C, OpenMP over the host cores."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    if threads:
        O.lib.orc_set_num_threads(threads)
    nthreads = O.lib.orc_num_threads()
    anum, aden = rational()
    theta, phi = inputs(0)
    Lo = O.lat(LX, LY, LT, LS, beta=BETA, am3=AM3)
    u = O.coef(Lo, theta)
    # the oracle times its own iteration loop: the allocation and filling of the 25
    # shift fields before it are not part of the sample
    O.multishift(Lo, u, AM, IMASS, anum[1:], aden, phi, RES, iters_sample)
    return O.lib.orc_last_loop_seconds() / iters_sample, nthreads


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


# ------------------------------------------------------------------ main
# ------------------------------------------------------------------ secondary workloads
def run_measurement(args):
    """Batched measurement solves: 24^2 x 24, Ls = 48, am = 0.02, 64 wall-noise
    sources + 4 spins x 4 point sources (Phi = M^dagger xi as measure_shamir
    builds them), congrad rule with res = 1e-8 (rescgm).  Compares one batched
    launch per operation (FP64, and FP32 corrections with FP64 defect
    correction) against one congrad call per source."""
    import torch
    import thirring
    from thirring import _lib
    L = _lib.lib()
    lx, ls, am, imass, res = 24, 48, 0.02, 1, 1e-8
    rng = np.random.default_rng(4)
    G = thirring.Lattice(lx, lx, lx, ls, beta=BETA)
    G.coef(np.asfortranarray(rng.standard_normal((lx, lx, lx, 3)) / np.sqrt(BETA), np.float32))
    nsrc = 80
    shp = (ls + 2, lx + 2, lx + 2, lx + 2, 4)
    xi = np.zeros(shp + (nsrc,), np.complex128, order="F")
    for k in range(64):
        d = k % 4
        s = 1 if d < 2 else ls
        xi[s, 1:-1, 1:-1, 1:-1, d, k] = rng.standard_normal((lx, lx, lx)) + 1j * rng.standard_normal((lx, lx, lx))
    pts = [(1, 1, 1), (7, 13, 5), (13, 7, 19), (19, 19, 11)]
    for j, (x0, y0, t0) in enumerate(pts):
        for d in range(4):
            xi[1 if d < 2 else ls, x0, y0, t0, d, 64 + 4 * j + d] = 1.0
    Phi = np.zeros_like(xi)
    for k in range(nsrc):
        Phi[..., k] = G.dslashd(np.asfortranarray(xi[..., k]), None, am, imass)
    n = 4 * ls * lx ** 3
    dev_phi = torch.zeros(nsrc * n, dtype=torch.complex128, device="cuda")
    for k in range(nsrc):
        i = Phi[1:-1, 1:-1, 1:-1, 1:-1, :, k]
        dev_phi[k * n:(k + 1) * n] = torch.from_numpy(np.ascontiguousarray(i.transpose(4, 3, 2, 1, 0)).ravel())
    out = {}
    for name, prec in (("fp64", 0), ("mixed_fp32", 2), ("mixed_bf16", 3)):
        best = None
        for rep in range(2):
            X = torch.zeros_like(dev_phi)
            its = np.zeros(nsrc, np.int32)
            outer = C.c_int(0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rc = L.thr_congrad_multi_dev(G.h, C.c_void_p(dev_phi.data_ptr()), C.c_void_p(X.data_ptr()), nsrc, res,
                                         am, imass, prec, its.ctypes.data_as(C.c_void_p), C.byref(outer))
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
        out[name] = {"s": round(best, 3), "rhs_per_s": round(nsrc / best, 2), "iters_mean": float(its.mean()),
                     "outer_rounds": outer.value, "rc": rc}
    # one congrad per source (FP64), on a sample of 8 sources
    t0 = time.perf_counter()
    for k in range(8):
        X = np.zeros(shp, np.complex128, order="F")
        G.congrad(np.asfortranarray(Phi[..., k]), X, res, am, imass)
    dt = (time.perf_counter() - t0) / 8 * nsrc
    out["sequential_fp64_congrad"] = {"s": round(dt, 3), "rhs_per_s": round(nsrc / dt, 2),
                                      "sample": "8 of 80 sources, scaled"}
    G.close()
    return {"workload": "measurement solves 24^2x24 Ls48, 80 sources, res 1e-8, am 0.02", "results": out}


def run_packed(args):
    """32 independent lattices, L ~ U{8..20}, T = L, Ls ~ U{8,12,..,32},
    beta ~ U[0.25, 0.5], seeds 1..32: one right-hand side each, solved
    together in one persistent launch per operation vs one congrad each."""
    import thirring
    rng = np.random.default_rng(2024)
    shapes, betas = [], []
    for i in range(32):
        lx = int(rng.integers(8, 21)) & ~1
        shapes.append((lx, lx, lx, int(rng.choice(range(8, 33, 4)))))
        betas.append(float(rng.uniform(0.25, 0.5)))
    am, imass, res = 0.02, 1, 1e-8
    pack = thirring.Pack(shapes)
    data = []
    for i, ((lx, ly, lt, ls), b) in enumerate(zip(shapes, betas)):
        r = np.random.default_rng(i + 1)
        th = np.asfortranarray(r.standard_normal((lx, ly, lt, 3)) / np.sqrt(b), np.float32)
        with thirring.Lattice(lx, ly, lt, ls, beta=b) as G:
            u = G.coef(th)
        phi = np.zeros((ls + 2, lx + 2, ly + 2, lt + 2, 4), np.complex128, order="F")
        sh = phi[1:-1, 1:-1, 1:-1, 1:-1, :].shape
        phi[1:-1, 1:-1, 1:-1, 1:-1, :] = r.standard_normal(sh) + 1j * r.standard_normal(sh)
        pack.upload(i, u, phi, np.zeros_like(phi))
        data.append((u, phi))
    out = {}
    for name, prec in (("fp64", 0), ("mixed_fp32", 2)):
        best = None
        for rep in range(2):
            pack.zero_x()
            t0 = time.perf_counter()
            its, outer = pack.congrad(res, am, imass, prec)
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
        out[name] = {"s": round(best, 3), "lattices_per_s": round(32 / best, 2), "iters_max": int(its.max()),
                     "outer_rounds": outer}
    t0 = time.perf_counter()
    for i, ((lx, ly, lt, ls), b) in enumerate(zip(shapes, betas)):
        with thirring.Lattice(lx, ly, lt, ls, beta=b) as G:
            G.set_links(data[i][0])
            X = np.zeros_like(data[i][1])
            G.congrad(data[i][1], X, res, am, imass)
    dt = time.perf_counter() - t0
    out["sequential_fp64_congrad"] = {"s": round(dt, 3), "lattices_per_s": round(32 / dt, 2)}
    pack.close()
    return {"workload": "32 packed lattices L 8..20, Ls 8..32, beta 0.25..0.5, res 1e-8", "shapes": shapes,
            "results": out}


def run_trajectory(args):
    """Config 1 on the GPU and on the host: 12^2 x 12, Ls = 16, Shamir, beta 0.3, am 0.05,
    imass 3, antiperiodic t, seeded Gaussian theta and site streams.
    (a) one congrad of M^dagger M x = Phi to res 1e-9 (measure_module.F90:9-140): the GPU
        (thr_congrad, FP64) against the oracle on the host cores, end to end;
    (b) one trajectory of 10 fixed MD steps, dt 0.05, with the reference's remez2/remez4
        (25 poles) and remez2g/remez4g (12 poles), rescga 1e-8, rescgg 1e-6, in the
        configurations: the plain FP64 GPU path (the reference's multishift loop
        structure, host-driven steps); FP64 batched with each MD step one CUDA graph; the
        mixed multishift for the action solves with FP64 guidance; the reference's
        single-precision guidance (spmd).  Each starts from the same theta and seed; its
        Delta H is compared with the oracle's FP64 trajectory (FP64 guidance) of the same
        start, whose time on the host cores is the CPU baseline of the trajectory."""
    import thirring
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    gold = os.path.join(REPO, "tests", "golden") + os.sep
    rat = thirring.remez_set(gold + "remez2", gold + "remez4", 25)
    ratg = thirring.remez_set(gold + "remez2g", gold + "remez4g", 12)
    lx, ls, beta, am, imass, dt, nstep = 12, 16, 0.3, 0.05, 3, 0.05, 10
    seed = 4139764973254.0
    rng = np.random.default_rng(1)
    th0 = np.asfortranarray(rng.standard_normal((lx, lx, lx, 3)) / np.sqrt(beta), np.float32)
    out = {}
    # (a) congrad to 1e-9 (--no-cpu: the GPU side only)
    Lo = O.lat(lx, lx, lx, ls, beta=beta, am3=AM3)
    u = O.coef(Lo, th0)
    phi = np.zeros((ls + 2, lx + 2, lx + 2, lx + 2, 4), np.complex128, order="F")
    sh = phi[1:-1, 1:-1, 1:-1, 1:-1, :].shape
    phi[1:-1, 1:-1, 1:-1, 1:-1, :] = rng.standard_normal(sh) + 1j * rng.standard_normal(sh)
    O.update_halo_5(Lo, phi)
    t0 = time.perf_counter()
    xr = O.spinor(Lo)
    it_ref = 0
    if not args.no_cpu:
        it_ref, _ = O.congrad(Lo, phi, xr, u, 1e-9, am, imass)
    cpu_cg = time.perf_counter() - t0
    with thirring.Lattice(lx, lx, lx, ls, beta=beta) as G:
        G.set_links(u)
        x = np.zeros_like(phi)
        G.congrad(phi, x, 1e-9, am, imass)  # warm-up (autotuner, graph)
        x = np.zeros_like(phi)
        t0 = time.perf_counter()
        it, _ = G.congrad(phi, x, 1e-9, am, imass)
        gpu_cg = time.perf_counter() - t0
    out["congrad_1e-9"] = {"gpu_s": round(gpu_cg, 4), "gpu_iterations": it,
                           "path": "thr_congrad with host Fortran-layout arrays (copies included)"}
    if not args.no_cpu:
        err = float(np.max(np.abs(O.interior(x) - O.interior(xr))) / np.max(np.abs(O.interior(xr))))
        out["congrad_1e-9"].update({"cpu_s": round(cpu_cg, 3), "cpu_iterations": it_ref,
                                    "cpu_cores": int(O.lib.orc_num_threads()), "speedup": round(cpu_cg / gpu_cg, 1),
                                    "max_rel_diff_vs_oracle": float("%.3g" % err)})
    # (b) trajectories
    ref, cpu_traj = None, None
    if not args.no_cpu:
        t0 = time.perf_counter()
        g = O.RNG(Lo, True).init(seed)
        th_ref = th0.copy(order="F")
        orat = O.rational(rat, ratg)
        ref = O.trajectory(Lo, g, th_ref, orat, nstep, dt, am, imass, 1e-8, 1e-6, 0, fixed_steps=nstep)
        cpu_traj = time.perf_counter() - t0
        out["oracle_fp64_trajectory"] = {"s": round(cpu_traj, 1), "dH": ref.dh, "accepted": ref.accepted,
                                         "cores": int(O.lib.orc_num_threads()), "cpu": cpu_model()}
    modes = (("plain_fp64_gpu", 0, 0, 0, False), ("fp64_batched_md_graph", 1, 0, 0, True),
             ("mixed_action_fp64_guidance", 1, 0, 2, True), ("spmd_fp32_guidance", 1, 1, 0, True))
    for name, algo, spmd, action, md_graph in modes:
        G = thirring.Lattice(lx, lx, lx, ls, beta=beta)
        G.set_solver(algo)
        G.set_remez(rat, ratg)
        G.set_residuals(1e-8, 1e-6, spmd)
        G.set_action_precision(action)
        times, res = [], None
        for rep in range(2):  # the first run settles buffers, autotuner and graphs
            G.init_random(seed)
            th = th0.copy(order="F")
            G.md_counters(reset=True)
            t1 = time.perf_counter()
            res = G.trajectory(th, nstep, dt, am, imass, fixed_steps=nstep)
            times.append(time.perf_counter() - t1)
        out[name] = {"s_per_traj": round(times[-1], 4), "traj_per_hr": round(3600 / times[-1], 1), "dH": res.dh,
                     "accepted": res.accepted, "md_step_graph": md_graph,
                     "iterations": {k: v for k, v in G.md_counters().items() if v}}
        if ref is not None:
            out[name]["dH_minus_oracle"] = float("%.3g" % (res.dh - ref.dh))
        G.close()
    base = out["plain_fp64_gpu"]["s_per_traj"]
    for name, *_ in modes:
        out[name]["speedup_vs_plain_fp64_gpu"] = round(base / out[name]["s_per_traj"], 2)
        if cpu_traj:
            out[name]["speedup_vs_oracle_cpu"] = round(cpu_traj / out[name]["s_per_traj"], 1)
    return {"workload": "config 1: 12^2x12 Ls16 Shamir, beta 0.3, am 0.05, imass 3; congrad to 1e-9; RHMC "
                        "trajectory of 10 MD steps dt 0.05, remez2/4 + remez2g/4g, rescga 1e-8, rescgg 1e-6",
            "results": out}


def run_trajectory48(args):
    """Config 5, one sample trajectory: 48^2 x 48, Ls = 48, beta 0.28, am 0.005, imass 3,
    50 fixed MD steps of dt 0.02 (--traj-steps), remez2/remez4 (25 poles) for the action
    and remez2g/remez4g (12 poles) for the guidance force; the reference's single-precision
    guidance solves (spmd) at rescgg 1e-6, the Hamiltonian and pseudofermion solves at
    rescga 1e-9 with the mixed multishift; each MD step after the first replayed as one
    CUDA graph; Gaussian theta, site streams.  One trajectory, not the 20 of the config:
    a full one takes about a quarter of an hour on one GPU.  Its Delta H cannot be compared
    with the oracle here (the oracle would take days at this size); config 1 carries that
    comparison.  --traj-mode plain runs the same trajectory on the plain FP64 GPU path (the
    reference's multishift loop structure, FP64 guidance and action solves, host-driven
    steps), for the speed-up over it (a short --traj-steps makes both comparable); ours64
    is this build's path with FP64 guidance solves, the like-for-like comparison."""
    import thirring
    gold = os.path.join(REPO, "tests", "golden") + os.sep
    rat = thirring.remez_set(gold + "remez2", gold + "remez4", 25)
    ratg = thirring.remez_set(gold + "remez2g", gold + "remez4g", 12)
    lx, ls, beta, am, dt = 48, 48, 0.28, 0.005, 0.02
    nstep = args.traj_steps
    G = thirring.Lattice(lx, lx, lx, ls, beta=beta)
    G.set_remez(rat, ratg)
    plain = args.traj_mode == "plain"
    if plain:
        G.set_solver(0)
        G.set_residuals(1e-9, 1e-6, 0)
    else:
        G.set_residuals(1e-9, 1e-6, 0 if args.traj_mode == "ours64" else 1)
        G.set_action_precision(thirring.MIXED_FP32)
    G.init_random(4139764973254.0)
    rng = np.random.default_rng(5)
    th = np.asfortranarray(rng.standard_normal((lx, lx, lx, 3)) / np.sqrt(beta), np.float32)
    G.md_counters(reset=True)
    with Clocks(0) as clk:
        t0 = time.perf_counter()
        r = G.trajectory(th, nstep, dt, am, 3, fixed_steps=nstep)
        t = time.perf_counter() - t0
    its = {k: v for k, v in G.md_counters().items() if v}
    G.close()
    how = ("plain FP64 GPU path: per-iteration multishift, FP64 guidance and action solves, host-driven steps"
           if plain else "%s guidance, mixed action solves, MD steps as CUDA graphs"
           % ("FP64" if args.traj_mode == "ours64" else "spmd"))
    return {"workload": "config 5 sample: one RHMC trajectory, 48^2x48 Ls48, beta 0.28, am 0.005, imass 3, "
                        "%d MD steps dt %g, %s" % (nstep, dt, how),
            "s_per_traj": round(t, 1), "traj_per_hr": round(3600 / t, 2), "dH": r.dh, "accepted": r.accepted,
            "steps": r.steps, "iterations": its, "clocks": clk.summary(), "sample": "1 trajectory"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="mixed", choices=["fp64", "sp", "mixed", "bf16"],
                    help="multishift precision: mixed (default) runs FP64 until |r| < 1e-8 |Phi|, then FP32 "
                         "stencils and residuals with FP64 shift fields")
    ap.add_argument("--workload", default="multishift",
                    choices=["multishift", "measurement", "packed", "trajectory", "trajectory48", "dslash",
                             "dslash_sweep", "aux_kernels", "overlap"],
                    help="secondary workloads print their own JSON line (not the headline contract)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-iters", type=int, default=50, help="multishift iterations in the CPU sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--lx", type=int, default=0, help="profiling case: lattice extent (all three directions)")
    ap.add_argument("--ls", type=int, default=0, help="profiling case: fifth-dimension extent")
    ap.add_argument("--poles", type=int, default=0, help="profiling case: number of poles")
    ap.add_argument("--max-iters", type=int, default=0,
                    help="profiling case: stop every solve after this many iterations (not a full solve)")
    ap.add_argument("--no-dslash", action="store_true")
    ap.add_argument("--traj-steps", type=int, default=50, help="trajectory48: MD steps of the sample trajectory")
    ap.add_argument("--traj-mode", default="ours", choices=["ours", "ours64", "plain"],
                    help="trajectory48: this build's path (default; ours64: with FP64 guidance solves) or the "
                         "plain FP64 GPU path")
    ap.add_argument("--sweep-l", default="", help="dslash_sweep: comma-separated lattice extents")
    ap.add_argument("--sweep-ls", default="", help="dslash_sweep: comma-separated fifth-dimension extents")
    ap.add_argument("--no-compare-plain", dest="compare_plain", action="store_false",
                    help="skip timing the plain FP64 path (reference loop structure)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    iters_for_cpu = FP64_ITERS_REF

    if args.lx or args.ls or args.poles:
        # a smaller (or larger) profiling case of the same solve; not the headline workload
        global LX, LY, LT, LS, NPOLE
        LX = LY = LT = args.lx or LX
        LS = args.ls or LS
        NPOLE = args.poles or NPOLE
    if args.workload == "dslash":
        lx, ls = args.lx or 48, args.ls or 48
        r = dslash_bandwidth(args, local_rank, lx, ls, args.steps, args.warmup)
        print(json.dumps({"workload": f"FP64 Shamir M and M^dagger, {lx}^2x{lx}, Ls={ls}, "
                                      f"{args.steps} launches each", "results": r}), flush=True)
        return
    if args.workload != "multishift":
        fn = {"measurement": run_measurement, "packed": run_packed, "trajectory": run_trajectory,
              "trajectory48": run_trajectory48, "overlap": run_overlap, "dslash_sweep": run_dslash_sweep,
              "aux_kernels": run_aux_kernels}[args.workload]
        print(json.dumps(fn(args)), flush=True)
        return

    if args.impl == "reference":
        if rank != 0:
            return
        t0 = time.perf_counter()
        per_iter = []
        nthreads = 0
        for _ in range(args.warmup + args.steps):
            s, nthreads = cpu_sample(max(1, args.cpu_iters // 2))  # loop time only, set-up excluded
            per_iter.append(s)
        timed = per_iter[args.warmup:]
        s_iter = float(np.mean(timed))
        iters = iters_for_cpu or 0
        value = 1.0 / (s_iter * iters) if iters else None
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": (s_iter * iters * 1e3) if iters else None,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded Gaussian theta, complex Gaussian source)",
                "config": workload_config(),
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                                 "sample": f"{max(1, args.cpu_iters // 2)} multishift iterations per step of the "
                                           f"same solve (the iteration loop timed, its set-up excluded), the solve "
                                           f"time projected to the {iters} iterations a full FP64 solve takes "
                                           f"({s_iter:.3f} s per iteration); {cpu_model()}"},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "wall_s": round(time.perf_counter() - t0, 1)}
        print(json.dumps(line), flush=True)
        return

    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))
    r = run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return
    iters = r["its"][-1]
    ms_step = r["ms"] / args.steps
    value = job_throughput(world, args.steps, r["ms"])
    peak, peak_kind = peaks()
    # per kernel: sampled launches give the mean duration and bytes per launch; the
    # kernel's time in the step is that mean times its launches
    kern = {}
    for name, p in r["prof"].items():
        if not p["sampled"] or p["ms"] <= 0:
            continue
        us = p["ms"] * 1e3 / p["sampled"]
        bpl = p["bytes"] / p["sampled"]
        kern[name] = {"launches": int(p["launches"]), "sampled": p["sampled"], "us_per_launch": round(us, 3),
                      "algorithmic_bytes_per_launch": round(bpl), "gbs": round(bpl / us / 1e3, 1),
                      "share_of_step": round(p["launches"] * us / 1e3 / ms_step, 4)}
    # dominant kernel of the timed region
    name = max(kern, key=lambda k: kern[k]["share_of_step"])
    k = kern[name]
    achieved = k["gbs"]
    traffic = ncu_traffic(name, k["algorithmic_bytes_per_launch"])
    roofline = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": peak_kind, "traffic": traffic,
                "traffic_source": ("not measured in this run: dram__bytes_read.sum + dram__bytes_write.sum per launch "
                                   "from the ncu capture summarised in profiles/ (profiles/roofline_traffic.txt)"
                                   if traffic is not None else None),
                "algorithmic_bytes_per_launch": k["algorithmic_bytes_per_launch"],
                "us_per_launch": k["us_per_launch"], "launches": k["launches"], "sampled_launches": k["sampled"],
                "share_of_step": k["share_of_step"]}
    other = kern
    cpu = None
    if not args.no_cpu:
        s_iter, nthreads = cpu_sample(args.cpu_iters)
        cpu_val = 1.0 / (s_iter * iters)
        cpu = {"value": cpu_val, "unit": UNIT, "cores": nthreads, "kind": "port",
               "sample": f"{args.cpu_iters} FP64 multishift iterations of the same solve (the iteration loop "
                         f"timed, set-up excluded: {s_iter:.3f} s per iteration), projected to the {iters} "
                         f"iterations the solve takes; {cpu_model()}"}
    e2e = None
    if r["e2e_ms"]:
        e2e = {"value": job_throughput(world, args.e2e_steps, r["e2e_ms"]), "unit": UNIT,
               "h2d_bytes_per_step": r["phi_bytes"], "d2h_bytes_per_step": r["phi_bytes"],
               "path": "thr_qmrherm (C ABI) with page-locked Fortran-layout host arrays"}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPES[args.mode],
            "data": "synthetic (seeded Gaussian theta, complex Gaussian source)",
            "config": workload_config(), "iterations": iters, "e2e": e2e, "roofline": roofline,
            "kernels": other, "cpu_baseline": cpu, "gpu_launches": r["launches"], "clocks": r["clocks"],
            "solve_s": ms_step / 1e3,
            "plain_fp64_gpu_solve_s": r["fp64_s"], "plain_fp64_gpu_iterations": r["fp64_iters"],
            "speedup_vs_plain_fp64_gpu": (r["fp64_s"] / (ms_step / 1e3)) if r["fp64_s"] else None,
            "batched_host_launched_solve_s": r["stream_s"],
            "batched_fp64_solve_s": r["fp64_batched_s"] if r["fp64_batched_s"] else ms_step / 1e3,
            "speedup_vs_batched_fp64": (r["fp64_batched_s"] / (ms_step / 1e3)) if r["fp64_batched_s"] else None,
            "accuracy": r["accuracy"],
            "autotune": r["tune"],
            "dslash_48x48x48_ls48_fp64": r["dslash"]}
    print(json.dumps(line), flush=True)


def workload_config():
    return {"workload": f"qmrherm multishift solve, {LX}^2x{LT} lattice, Ls={LS}, Shamir, {NPOLE} poles "
                        f"log-spaced 1e-5..1e2, am={AM}, imass={IMASS}, beta={BETA}, res={RES}",
            "lattice": [LX, LY, LT, LS], "poles": NPOLE, "l2_flush": "not needed: working set 3.4 GB > L2",
            "parallelism": "replicas (one lattice per GPU)"}


if __name__ == "__main__":
    main()
