"""ctypes binding of the CPU restatement (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by the test suite, the smoke check and the
CPU-baseline leg of the benchmark, never by the product package.

Arrays are numpy arrays in the reference's Fortran layout (order='F'), halos
included, exactly as the Fortran routines declare them (see
thirring_oracle.h for the shapes).
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load():
    if not os.path.exists(_LIB):
        build()
    return C.CDLL(_LIB)


lib = _load()


class Lat(C.Structure):
    _fields_ = [("lx", C.c_int), ("ly", C.c_int), ("lt", C.c_int), ("ls", C.c_int),
                ("kernel", C.c_int), ("ndiag", C.c_int), ("am3", C.c_float),
                ("beta", C.c_float), ("ibound", C.c_int), ("nf", C.c_int),
                ("strict_sums", C.c_int)]


class Rational(C.Structure):
    _fields_ = [("ndiag", C.c_int), ("ndiagg", C.c_int)] + [
        (n, C.POINTER(C.c_double)) for n in (
            "anum2", "aden2", "bnum2", "bden2", "anum4", "aden4", "bnum4", "bden4",
            "anum2g", "aden2g", "bnum2g", "bden2g", "anum4g", "aden4g", "bnum4g", "bden4g")]


class TrajResult(C.Structure):
    _fields_ = [("h0", C.c_double), ("h1", C.c_double), ("dh", C.c_double), ("ds", C.c_double),
                ("s0", C.c_double), ("s1", C.c_double), ("accepted", C.c_int), ("steps", C.c_int),
                ("y", C.c_float)]


class Counts(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("ancg", "ancgpv", "ancgf", "ancgfpv", "ancgh",
                                          "ancghpv", "ancgpf", "ancgpfpv")]


def P(a):
    """numpy array -> void pointer (must be contiguous in Fortran order)."""
    if a is None:
        return None
    assert a.flags.f_contiguous or a.flags.c_contiguous
    return a.ctypes.data_as(C.c_void_p)


def lat(lx, ly, lt, ls, kernel=0, ndiag=25, am3=1.0, beta=0.4, ibound=-1, nf=1, strict_sums=0):
    return Lat(lx, ly, lt, ls, kernel, ndiag, am3, beta, ibound, nf, strict_sums)


def spinor(L, dtype=np.complex128):
    return np.zeros((L.ls + 2, L.lx + 2, L.ly + 2, L.lt + 2, 4), dtype=dtype, order="F")


def links(L):
    return np.zeros((L.lx + 2, L.ly + 2, L.lt + 2, 3), dtype=np.complex128, order="F")


def field3(L, dtype=np.float64):
    return np.zeros((L.lx, L.ly, L.lt, 3), dtype=dtype, order="F")


def ps_field(L):
    return np.zeros((L.lx + 2, L.ly + 2, L.lt + 2, 2), dtype=np.float32, order="F")


def shift_out(L, ndiag=None):
    return np.zeros((L.ls, L.lx, L.ly, L.lt, 4, ndiag or L.ndiag), dtype=np.complex128, order="F")


def interior(a):
    """Interior of a halo'd spinor (drops the first four halos)."""
    return a[1:-1, 1:-1, 1:-1, 1:-1, :]


_v = C.c_void_p
_L = C.POINTER(Lat)
for name, res, args in [
    ("orc_update_halo_5", None, [_L, _v]),
    ("orc_update_halo_4", None, [_L, C.c_int, _v]),
    ("orc_update_halo_4_real", None, [_L, C.c_int, _v]),
    ("orc_dwilson", None, [_L, _v, _v, _v, C.c_float]),
    ("orc_coef", None, [_L, _v, _v]),
    ("orc_dslash", None, [_L, _v, _v, _v, C.c_float, C.c_int]),
    ("orc_dslashd", None, [_L, _v, _v, _v, C.c_float, C.c_int]),
    ("orc_dslash_sp", None, [_L, _v, _v, _v, C.c_float, C.c_int]),
    ("orc_dslashd_sp", None, [_L, _v, _v, _v, C.c_float, C.c_int]),
    ("orc_dirac_operator", None, [_L, _v, _v, _v, C.c_float, C.c_int]),
    ("orc_congrad", C.c_int, [_L, _v, _v, _v, C.c_float, C.c_float, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    ("orc_multishift_solver", None, [_L, _v, C.c_float, C.c_int, C.c_int, _v, _v, _v, _v, C.c_float, C.c_int,
                                     C.POINTER(C.c_int), _v]),
    ("orc_multishift_solver_sp", None, [_L, _v, C.c_float, C.c_int, C.c_int, _v, _v, _v, _v, C.c_float, C.c_int,
                                        C.POINTER(C.c_int), _v]),
    ("orc_derivs", None, [_L, _v, _v, C.c_double, C.c_int, C.c_float, C.c_int, _v]),
    ("orc_qmrherm", C.c_int, [_L, _v, _v, _v, C.c_float, C.POINTER(C.c_int), C.c_float, C.c_int, _v, _v, C.c_int,
                              C.c_int, C.c_int, C.c_int, _v, _v, _v, _v]),
    ("orc_rng_create", _v, [_L, C.c_int]),
    ("orc_rng_destroy", None, [_v]),
    ("orc_init_random", C.c_int, [_v, C.c_double]),
    ("orc_rano", C.c_float, [_v, C.c_int, C.c_int, C.c_int]),
    ("orc_dranf", C.c_double, [_v, C.c_int, C.c_int, C.c_int]),
    ("orc_rranget", C.c_double, [_v, C.c_int, C.c_int, C.c_int]),
    ("orc_gauss0", None, [_L, _v, _v]),
    ("orc_gaussp", None, [_L, _v, _v]),
    ("orc_read_remez_file", C.c_int, [C.c_char_p, C.c_int, _v, _v, _v, _v]),
    ("orc_starting_state", None, [_L, _v, _v, _v, _v, _v, _v]),
    ("orc_initialise_phi", C.c_int, [_L, _v, _v, C.POINTER(Rational), _v, C.c_float, C.c_int, C.c_float, C.c_int,
                                     C.POINTER(Counts)]),
    ("orc_initialise_pp", None, [_L, _v, _v]),
    ("orc_force", C.c_int, [_L, _v, _v, C.POINTER(Rational), _v, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int,
                            _v, C.POINTER(Counts)]),
    ("orc_hamilton", C.c_int, [_L, _v, _v, _v, C.POINTER(Rational), _v, C.c_float, C.c_float, C.c_int, C.c_int,
                               C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                               C.POINTER(C.c_double), C.POINTER(Counts)]),
    ("orc_evolve_theta_pp", C.c_int, [_L, _v, _v, _v, _v, C.POINTER(Rational), _v, C.c_int, C.c_float, C.c_float,
                                      C.c_float, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), _v,
                                      C.POINTER(Counts)]),
    ("orc_trajectory", C.c_int, [_L, _v, _v, C.POINTER(Rational), C.c_int, C.c_float, C.c_float, C.c_int, C.c_float,
                                 C.c_float, C.c_int, C.c_int, C.c_int, C.POINTER(TrajResult), C.POINTER(Counts)]),
    ("orc_zolo_coeffs", None, [C.c_int, C.c_double, C.c_double, _v]),
    ("orc_odslash", None, [_L, _v, _v, _v, C.c_float, C.c_int, _v]),
    ("orc_odslashd", None, [_L, _v, _v, _v, C.c_float, C.c_int, _v]),
    ("orc_congrad_o", C.c_int, [_L, _v, _v, _v, C.c_float, C.c_float, C.c_int, _v, C.c_int, C.POINTER(C.c_int)]),
    ("orc_num_threads", C.c_int, []),
    ("orc_last_loop_seconds", C.c_double, []),
    ("orc_set_num_threads", None, [C.c_int]),
]:
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args


# ---------------------------------------------------------------- wrappers
def starting_state(L, Phi=True, u=True, R=False, X=False, dSdpi=False, Phi0=False):
    """tests/test_utils.F90:35-151 analytic state; returns dict of arrays."""
    out = {}
    out["Phi"] = spinor(L) if Phi else None
    out["u"] = links(L) if u else None
    out["R"] = spinor(L) if R else None
    out["X"] = spinor(L) if X else None
    out["dSdpi"] = field3(L) if dSdpi else None
    out["Phi0"] = (np.zeros((L.ls + 2, L.lx + 2, L.ly + 2, L.lt + 2, 4, 25), np.complex128, order="F")
                   if Phi0 else None)
    lib.orc_starting_state(C.byref(L), P(out["Phi"]), P(out["u"]), P(out["R"]), P(out["X"]),
                           P(out["dSdpi"]), P(out["Phi0"]))
    return out


def dslash(L, R, u, am, imass):
    Phi = spinor(L)
    lib.orc_dslash(C.byref(L), P(Phi), P(R), P(u), am, imass)
    return Phi


def dslashd(L, R, u, am, imass):
    Phi = spinor(L)
    lib.orc_dslashd(C.byref(L), P(Phi), P(R), P(u), am, imass)
    return Phi


def dirac_operator(L, X, u, am, imass):
    """M^dagger M X with halos refreshed (inverter_utils.F90:20-54)."""
    out = spinor(L)
    lib.orc_dirac_operator(C.byref(L), P(out), P(X), P(u), am, imass)
    return out


def zolo_coeffs(n, lmin=0.1, lmax=5.0):
    """coeffs(1..n) of prepZolo (measure_OWilson.F90:169-188; defaults as there)."""
    c = np.zeros(n)
    lib.orc_zolo_coeffs(n, lmin, lmax, P(c))
    return c


def zolo_sign(coeffs, lmin, x):
    """The sign function from the roots 1/coeffs (zsgnrts, ZOLO/zolomodule.f:253-270)."""
    t = np.ones_like(np.asarray(x, dtype=float))
    for r in 1.0 / np.asarray(coeffs):
        t = t * (r - x) / (r + x)
    return (1 - t) / (1 + t)


def odslash(L, R, u, am, imass, coeffs):
    Phi = spinor(L)
    lib.orc_odslash(C.byref(L), P(Phi), P(R), P(u), am, imass, P(np.ascontiguousarray(coeffs, np.float64)))
    return Phi


def odslashd(L, R, u, am, imass, coeffs):
    Phi = spinor(L)
    lib.orc_odslashd(C.byref(L), P(Phi), P(R), P(u), am, imass, P(np.ascontiguousarray(coeffs, np.float64)))
    return Phi


def congrad_o(L, Phi, u, res, am, imass, coeffs, niterc=None):
    """congradO (measure_OWilson.F90:190-268): returns (X, itercg, iterations)."""
    X = spinor(L)
    it = C.c_int(0)
    niterc = niterc if niterc is not None else L.ls * L.lx * L.ly * L.lt
    itercg = lib.orc_congrad_o(C.byref(L), P(Phi), P(X), P(u), res, am, imass,
                               P(np.ascontiguousarray(coeffs, np.float64)), niterc, C.byref(it))
    return X, itercg, it.value


def update_halo_5(L, a):
    lib.orc_update_halo_5(C.byref(L), P(a))
    return a


def update_halo_4(L, a, n=3):
    lib.orc_update_halo_4(C.byref(L), n, P(a))
    return a


def coef(L, theta):
    u = links(L)
    lib.orc_coef(C.byref(L), P(u), P(np.asfortranarray(theta, np.float32)))
    return u


def congrad(L, Phi, X, u, res, am, imass, niterc=None):
    it = C.c_int(0)
    niterc = niterc if niterc is not None else L.ls * L.lx * L.ly * L.lt
    itercg = lib.orc_congrad(C.byref(L), P(Phi), P(X), P(u), res, am, imass, niterc, C.byref(it))
    return itercg, it.value


def multishift(L, u, am, imass, anum, aden, inp, res, maxcg, sp=False):
    nq = len(aden)
    out = shift_out(L)
    ret = C.c_int(0)
    cgr = np.zeros(nq, np.int32)
    fn = lib.orc_multishift_solver_sp if sp else lib.orc_multishift_solver
    fn(C.byref(L), P(u), am, imass, nq, P(np.ascontiguousarray(aden, np.float64)),
       P(np.ascontiguousarray(anum, np.float64)), P(out), P(inp), res, maxcg, C.byref(ret), P(cgr))
    return out, ret.value, cgr


def qmrherm(L, u, Phi, res, am, imass, anum, aden, iflag, use_sp=False, max_iters=50000,
            dSdpi=None, Phi0=None):
    """anum has ndiagq+1 entries; returns (x, itercg, cg_returns, rc)."""
    nq = len(aden)
    x = spinor(L)
    it = C.c_int(0)
    cgr = np.zeros(nq, np.int32)
    if dSdpi is None:
        dSdpi = field3(L)
    if Phi0 is None:
        Phi0 = np.zeros((L.ls + 2, L.lx + 2, L.ly + 2, L.lt + 2, 4, L.ndiag), np.complex128, order="F")
    rc = lib.orc_qmrherm(C.byref(L), P(u), P(Phi), P(x), res, C.byref(it), am, imass,
                         P(np.ascontiguousarray(anum, np.float64)), P(np.ascontiguousarray(aden, np.float64)),
                         nq, iflag, int(use_sp), max_iters, P(cgr), P(dSdpi), P(Phi0), None)
    return x, it.value, cgr, rc


def derivs(L, R, X2, anum, iflag, am, imass, dSdpi):
    lib.orc_derivs(C.byref(L), P(R), P(X2), anum, iflag, am, imass, P(dSdpi))
    return dSdpi


class RNG:
    def __init__(self, L, site=True):
        self.L = L
        self.h = lib.orc_rng_create(C.byref(L), int(site))

    def init(self, seed):
        rc = lib.orc_init_random(self.h, seed)
        assert rc == 0
        return self

    def rano(self, ix=1, iy=1, it=1):
        return lib.orc_rano(self.h, ix, iy, it)

    def rranget(self, ix=1, iy=1, it=1):
        return lib.orc_rranget(self.h, ix, iy, it)

    def gauss0(self):
        ps = ps_field(self.L)
        lib.orc_gauss0(C.byref(self.L), self.h, P(ps))
        return ps

    def gaussp(self):
        ps = ps_field(self.L)
        lib.orc_gaussp(C.byref(self.L), self.h, P(ps))
        return ps

    def __del__(self):
        try:
            lib.orc_rng_destroy(self.h)
        except Exception:
            pass


def read_remez(path, n):
    a = np.zeros(n + 1)
    b = np.zeros(n + 1)
    ad = np.zeros(n)
    bd = np.zeros(n)
    rc = lib.orc_read_remez_file(path.encode(), n, P(a), P(b), P(ad), P(bd))
    assert rc == 0, path
    return a, ad, b, bd


# ---------------------------------------------------------------- RHMC
_RKEYS = ("anum2", "aden2", "bnum2", "bden2", "anum4", "aden4", "bnum4", "bden4")


def rational(rat, ratg):
    """orc_rational from the remez / remezg dicts (see thirring.remez_set)."""
    r = Rational()
    r.ndiag = len(rat["aden2"])
    r.ndiagg = len(ratg["aden2"])
    keep = []
    for suffix, d in (("", rat), ("g", ratg)):
        for k in _RKEYS:
            a = np.ascontiguousarray(d[k], np.float64)
            keep.append(a)
            setattr(r, k + suffix, a.ctypes.data_as(C.POINTER(C.c_double)))
    r._keep = keep
    return r


def force(L, u, theta, rat, Phi, res1, am, imass, use_sp, max_iters=50000):
    dS = field3(L)
    cnt = Counts()
    rc = lib.orc_force(C.byref(L), P(u), P(np.asfortranarray(theta, np.float32)), C.byref(rat), P(Phi), res1, am,
                       imass, int(use_sp), max_iters, P(dS), C.byref(cnt))
    assert rc == 0
    return dS


def hamilton(L, u, theta, pp, rat, Phi, res2, am, imass, max_iters=50000):
    v = [C.c_double(0) for _ in range(4)]
    cnt = Counts()
    rc = lib.orc_hamilton(C.byref(L), P(u), P(np.asfortranarray(theta, np.float32)),
                          P(np.asfortranarray(pp, np.float32)), C.byref(rat), P(Phi), res2, am, imass, max_iters,
                          *[C.byref(x) for x in v], C.byref(cnt))
    assert rc == 0
    return tuple(x.value for x in v)


def initialise_phi(L, g, u, rat, am, imass, rescga=1e-8):
    Phi = spinor(L)
    cnt = Counts()
    rc = lib.orc_initialise_phi(C.byref(L), g.h, P(u), C.byref(rat), P(Phi), am, imass, rescga, 50000, C.byref(cnt))
    assert rc == 0
    return Phi


def initialise_pp(L, g):
    pp = field3(L, np.float32)
    lib.orc_initialise_pp(C.byref(L), g.h, P(pp))
    return pp


def trajectory(L, g, theta, rat, iterl, dt, am, imass, rescga, rescgg, use_sp, fixed_steps=0):
    r = TrajResult()
    cnt = Counts()
    rc = lib.orc_trajectory(C.byref(L), g.h, P(theta), C.byref(rat), iterl, dt, am, imass, rescga, rescgg,
                            int(use_sp), 50000, fixed_steps, C.byref(r), C.byref(cnt))
    assert rc == 0
    return r


# ---------------------------------------------------------------- measurement
def _with_kernel(L, kernel):
    M = Lat()
    C.memmove(C.byref(M), C.byref(L), C.sizeof(Lat))
    M.kernel = kernel
    return M


def measure_solves(ls, imass, kernel_meas):
    """The solves of one noise in the reference's order, 0-based:
    (wall noise 0 = ps / 1 = pt, source s, source spin, source sign,
     contraction s, contraction spin, post-projection 0 / 1 = P+ / 2 = P-, part 0 / 1).
    measure_shamir: measure_module.F90:221-334; measure_wilson: :495-590."""
    out = []
    if kernel_meas == 0:
        for i in range(2):
            if imass != 5:
                out.append((0, 0, i, 1.0, ls - 1, i, 0, 0))
                out.append((1, ls - 1, i + 2, 1.0, 0, i + 2, 0, 1))
            else:
                out.append((0, 0, i, -1.0, 0, i + 2, 0, 0))
                out.append((1, ls - 1, i + 2, -1.0, ls - 1, i, 0, 1))
    else:
        for i in range(4):
            out.append((0, 0, i, 1.0, ls - 1, i, 1, 0))
        for i in range(4):
            out.append((1, ls - 1, i, 1.0, 0, i, 2, 1))
    return out


def measure(L, g, u, res, am, imass, kernel_meas=0, knoise=10):
    """measure(psibarpsi, res, aviter, am, imass), measure_module.F90:142-162,
    with the measurement kernel chosen at run time (MEASURE_SHAMIR -> 0,
    MEASURE_WILSON -> 1):
      measure_shamir :170-423 -- per noise gauss0(ps), gauss0(pt); for
        idsource = 1, 2 a source on the wall s = 1 (from ps) and one on s = Ls
        (from pt); Phi = M^dagger xi with the measurement kernel's dslashd
        (:246), congrad(Phi) on the generation kernel with the source as the
        initial guess (vector::X is xi, :173); psibarpsi1/2 += sum conj(eta) *
        solution on the opposite wall (FP64 complex);
      measure_wilson :431-670 -- idsource = 1..4 on each wall, and before the
        contraction the wall slice of the solution becomes
        DWilson(P xi, -am3) - P xi with P = P+ (spins 1,2) at s = Ls and
        P- (spins 3,4) at s = 1.
    Returns psibarpsi, susclsing, aviter (float32 as in the reference), the
    per-noise (psibarpsi1, psibarpsi2) and each solve's itercg."""
    Lm = _with_kernel(L, kernel_meas)
    kvol = L.lx * L.ly * L.lt
    pbp = np.zeros(knoise)
    parts = []
    its = []
    it_total = 0
    for n in range(knoise):
        noise = [g.gauss0(), g.gauss0()]
        etas = [p[1:-1, 1:-1, 1:-1, 0].astype(np.float64) + 1j * p[1:-1, 1:-1, 1:-1, 1].astype(np.float64)
                for p in noise]
        acc = [0j, 0j]
        for (w, s_src, d_src, sign, s_c, d_c, post, part) in measure_solves(L.ls, imass, kernel_meas):
            xi = spinor(L)
            xi[s_src + 1, 1:-1, 1:-1, 1:-1, d_src] = sign * etas[w]
            update_halo_5(L, xi)
            Phi = update_halo_5(L, dslashd(Lm, xi, u, am, imass))
            itercg, _ = congrad(L, Phi, xi, u, res, am, imass)
            it_total += itercg
            its.append(itercg)
            if post:
                isl = np.zeros((L.lx + 2, L.ly + 2, L.lt + 2, 4), np.complex128, order="F")
                dd = (0, 1) if post == 1 else (2, 3)
                for d in dd:
                    isl[:, :, :, d] = xi[s_c + 1, :, :, :, d]
                osl = np.zeros_like(isl)
                lib.orc_dwilson(C.byref(L), P(osl), P(isl), P(u), -L.am3)
                wall = (osl - isl)[1:-1, 1:-1, 1:-1, d_c]
            else:
                wall = xi[s_c + 1, 1:-1, 1:-1, 1:-1, d_c]
            acc[part] = acc[part] + np.sum(np.conj(etas[w]) * wall)
        p1, p2 = acc
        if imass == 1:
            p1, p2 = p1 / kvol, p2 / kvol
        elif imass == 3:
            p1, p2 = -1j * p1 / kvol, 1j * p2 / kvol
        else:
            p1, p2 = -1j * p1 / kvol, -1j * p2 / kvol
        pbp[n] = (p1 + p2).real
        parts.append((p1, p2))
    psibarpsi = np.float32(np.sum(pbp))
    sus = np.float32(0.0)
    for n in range(knoise):
        sus = np.float32(sus + np.float32(np.sum(pbp[n] * pbp[n + 1:])))
    psibarpsi = np.float32(psibarpsi / np.float32(knoise))
    sus = np.float32(np.float32(2 * kvol) * sus / np.float32(knoise * (knoise - 1)))
    aviter = np.float32(np.float32(it_total) / np.float32(4 * knoise))
    return dict(psibarpsi=float(psibarpsi), susclsing=float(sus), aviter=float(aviter), parts=parts,
                pbp=pbp, itercg=its)


def permm(L, R, dagger):
    """PermM (measure_OWilson.F90:546-576) on halo'd 5D arrays, slices 1..Ls:
    PR(l) = P- R(l) + P+ R(l+1) with R(Ls+1) -> R(1); dagger: P+ R(l-1) with
    R(0) -> R(Ls).  P+ = spins 1,2 (Pplus :524-533), P- = spins 3,4 (:535-544)."""
    Ls = L.ls
    PR = spinor(L)
    PR[1:Ls + 1, :, :, :, 2:4] = R[1:Ls + 1, :, :, :, 2:4]
    for l in range(1, Ls + 1):
        if not dagger:
            tgt = Ls if l == 1 else l - 1
        else:
            tgt = 1 if l == Ls else l + 1
        PR[tgt, :, :, :, 0:2] += R[l, :, :, :, 0:2]
    return PR


def iddw(L, u, R, mass, imass, coeffs, respbp):
    """IDDW (measure_OWilson.F90:270-289): congradO(odslashd R) = DDW^-1 R; (X, itercg)."""
    IDR = update_halo_5(L, odslashd(L, R, u, mass, imass, coeffs))
    X, itc, _ = congrad_o(L, IDR, u, respbp, mass, imass, coeffs)
    return X, itc


def kddw(L, u, R, bmass, imass, coeffs, respbp):
    """KDDW (:342-367): PermM^dag . DDW(1)^-1 . DDW(bmass) . PermM R."""
    DR = update_halo_5(L, odslash(L, permm(L, R, False), u, bmass, imass, coeffs))
    X, _ = iddw(L, u, DR, 1.0, 1, coeffs, respbp)
    return permm(L, X, True)


def ikddw(L, u, R, bmass, imass, coeffs, respbp):
    """IKDDW (:369-393): PermM^dag . DDW(bmass)^-1 . DDW(1) . PermM R; (result, itercg)."""
    DR = update_halo_5(L, odslash(L, permm(L, R, False), u, 1.0, 1, coeffs))
    X, itc = iddw(L, u, DR, bmass, imass, coeffs, respbp)
    return permm(L, X, True), itc


def measure_ow(L, g, u, respbp, bmass, imass, coeffs, knoise=10):
    """measure_wilsonKDDW (measure_OWilson.F90:646-673, the MEASURE_OWILSON branch
    of measure, measure_module.F90:158-160): per noise evalSingleCondNoise_KDDW4
    (:704-757) -- for idx = 1..4 gauss0(ps), eta = cmplx(ps) on spin idx, IKDDW4
    (:462-478: eta on the slice s = 1 of a 5D field, IKDDW :369-393 = PermM^dag .
    IDDW(bmass) . odslash(mass 1, imass 1) . PermM, with IDDW :270-289 = congradO
    (respbp) of odslashd(bmass)), trace conj(eta) (IKDDW4 eta - eta) over spin idx
    divided by 1 - bmass (imass 1) or (-bmass, +-1) (imass 3), / kvol.
    psibarpsi = sum Re(pbp) / knoise, susclsing as output_OW (:674-702), aviter 0."""
    kvol = L.lx * L.ly * L.lt
    vpbp, cpbp, its = [], [], []
    for n in range(knoise):
        pbp = 0j
        for idx in range(4):
            ps = g.gauss0()
            eta = np.zeros((L.lx + 2, L.ly + 2, L.lt + 2, 4), np.complex128, order="F")
            eta[:, :, :, idx] = ps[:, :, :, 0].astype(np.float64) + 1j * ps[:, :, :, 1].astype(np.float64)
            R5 = spinor(L)
            R5[1] = eta  # IKDDW4 (:462-478)
            DR5, itc = ikddw(L, u, R5, bmass, imass, coeffs, respbp)
            its.append(itc)
            DR4 = DR5[1]
            tr = np.sum((np.conj(eta) * (DR4 - eta))[1:-1, 1:-1, 1:-1, idx])
            if imass == 1:
                denom = complex(float(np.float32(1.0) - np.float32(bmass)), 0.0)
            else:
                denom = complex(-float(np.float32(bmass)), 1.0 if idx < 2 else -1.0)
            pbp += tr / denom
        pbp = pbp / kvol
        cpbp.append(pbp)
        vpbp.append(pbp.real)
    vp = np.array(vpbp)
    psibarpsi = np.float32(np.sum(vp) / knoise)
    sus = np.float32(0.0)
    for n in range(knoise):
        sus = np.float32(sus + np.float32(np.sum(vp[n] * vp[n + 1:])))
    sus = np.float32(np.float32(2 * kvol) * sus / np.float32(knoise * (knoise - 1)))
    return dict(psibarpsi=float(psibarpsi), susclsing=float(sus), aviter=0.0, cpbp=cpbp, itercg=its)


def _wall_props(L, u, xi_src, res, am, imass):
    """measure_module.F90:811-826 (and :1162-1177): Phi = M^dagger xi, the initial
    guess M^dagger Phi, congrad; returns (itercg, solution)."""
    Phi = update_halo_5(L, dslashd(L, xi_src, u, am, imass))
    X = update_halo_5(L, dslashd(L, Phi, u, am, imass))
    itercg, _ = congrad(L, Phi, X, u, res, am, imass)
    return itercg, X


def meson(L, g, u, res, am, imass, nsource=5):
    """meson(res, itercg, aviter, am, imass), measure_module.F90:684-1085 with
    SITE_RANDOM source positions (three rano draws at site (1,1,1) per source)
    and nsmear = 0: point sources on the wall s = 1, spins 3 and 4; propagators
    to s = 1 (spins 1,2) and s = Ls (spins 3,4); for imass != 1 also with -am.
    Returns cpm, cmm (real(dp)), cpmn, cmmn (complex(dp)) per time separation,
    chim, the last itercg and aviter."""
    lx, ly, lt, ls = L.lx, L.ly, L.lt, L.ls
    cpm = np.zeros(lt); cmm = np.zeros(lt)
    cpmn = np.zeros(lt, complex); cmmn = np.zeros(lt, complex)
    it_total = 0
    itercg = 0
    for _ in range(nsource):
        ix = int(np.float32(lx) * np.float32(g.rano(1, 1, 1))) + 1
        iy = int(np.float32(lx) * np.float32(g.rano(1, 1, 1))) + 1  # ksize for x and y
        itt0 = int(np.float32(lt) * np.float32(g.rano(1, 1, 1))) + 1
        p00 = np.zeros((lx, ly, lt, 2, 2), complex); p0L = np.zeros_like(p00)
        p00n = np.zeros_like(p00); p0Ln = np.zeros_like(p00)
        for k, ids in enumerate((3, 4)):
            xi = spinor(L)
            xi[1, ix, iy, itt0, ids - 1] = 1.0
            update_halo_5(L, xi)
            itercg, X = _wall_props(L, u, xi, res, am, imass)
            it_total += itercg
            p00[..., k, :] = X[1, 1:-1, 1:-1, 1:-1, 0:2]
            p0L[..., k, :] = X[ls, 1:-1, 1:-1, 1:-1, 2:4]
            if imass != 1:
                itercg, Xn = _wall_props(L, u, xi, res, -am, imass)
                it_total += itercg
                p00n[..., k, :] = Xn[1, 1:-1, 1:-1, 1:-1, 0:2]
                p0Ln[..., k, :] = Xn[ls, 1:-1, 1:-1, 1:-1, 2:4]
            else:
                p00n[..., k, :] = p00[..., k, :]
                p0Ln[..., k, :] = p0L[..., k, :]
        for it in range(lt):
            t = (itt0 - 1 + it) % lt
            cpm[it] += np.sum(np.abs(p00[:, :, t]) ** 2)
            cpmn[it] += np.sum(p00[:, :, t] * np.conj(p00n[:, :, t]))
            cmm[it] += np.sum(np.abs(p0L[:, :, t]) ** 2)
            cmmn[it] += np.sum(p0L[:, :, t] * np.conj(p0Ln[:, :, t]))
    cpm /= nsource; cmm /= nsource; cpmn /= nsource; cmmn /= nsource
    chim = 0.0
    for it in range(lt):
        chim += 2 * (cpm[it] + cmm[it])
    aviter = np.float32(np.float32(it_total) / np.float32(2 * nsource))
    return dict(cpm=cpm, cmm=cmm, cpmn=cpmn, cmmn=cmmn, chim=chim, itercg=itercg, aviter=float(aviter))


# 2 gamma(3, d) (gammamatrices.F90: mu = 3 row, already times akappa = 1/2 there)
_GAMVAL3 = {3: 0.5j, 4: -0.5j}
_GAMIN3 = {3: 1, 4: 2}


def fermion(L, g, u, res, am, imass, nsource=5, ibound=-1):
    """fermion(res, itercg, aviter, am, imass), measure_module.F90:1100-1376 with
    SITE_RANDOM source times: wall sources 1/ksize2 on a whole time slice at
    s = 1, spins 3 and 4; cferm1(t) = sum isign akappa prop0L(.,t,d,d),
    cferm2(t) = sum isign gamval(3,d) prop00(.,t,d,gamin(3,d)), isign = ibound
    across the time boundary.  Returns cferm1, cferm2, the last itercg, aviter."""
    lx, ly, lt, ls = L.lx, L.ly, L.lt, L.ls
    cf1 = np.zeros(lt, complex); cf2 = np.zeros(lt, complex)
    it_total = 0
    itercg = 0
    for _ in range(nsource):
        itt0 = int(np.float32(lt) * np.float32(g.rano(1, 1, 1))) + 1
        p00 = {}; p0L = {}
        for ids in (3, 4):
            xi = spinor(L)
            # cmplx(1.0, 0.0) / ksize2: a default-real complex, widened
            xi[1, 1:-1, 1:-1, itt0, ids - 1] = float(np.float32(1.0) / np.float32(lx * lx))
            update_halo_5(L, xi)
            itercg, X = _wall_props(L, u, xi, res, am, imass)
            it_total += itercg
            p00[ids] = X[1, 1:-1, 1:-1, 1:-1, :]
            p0L[ids] = X[ls, 1:-1, 1:-1, 1:-1, :]
        t1 = np.zeros(lt, complex); t2 = np.zeros(lt, complex)
        for idd in (3, 4):
            for it in range(lt):
                itt = (itt0 - 1 + it) % lt + 1
                isign = 1 if itt >= itt0 else ibound
                t1[it] += isign * 0.5 * np.sum(p0L[idd][:, :, itt - 1, idd - 1])
        for idd in (3, 4):
            for it in range(lt):
                itt = (itt0 - 1 + it) % lt + 1
                isign = 1 if itt >= itt0 else ibound
                t2[it] += isign * _GAMVAL3[idd] * np.sum(p00[idd][:, :, itt - 1, _GAMIN3[idd] - 1])
        cf1 += t1; cf2 += t2
    cf1 /= nsource; cf2 /= nsource
    aviter = np.float32(np.float32(it_total) / np.float32(2 * nsource))
    return dict(cferm1=cf1, cferm2=cf2, itercg=itercg, aviter=float(aviter))
