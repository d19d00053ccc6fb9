"""Reference-shaped API over the C ABI.

Array shapes (numpy, order='F'), as declared in the reference:
  spinor  complex128 (Ls+2, Lx+2, Ly+2, Lt+2, 4)      dirac.F90:13-15
  links   complex128 (Lx+2, Ly+2, Lt+2, 3)            trial.F90:6
  theta   float32    (Lx, Ly, Lt, 3)                  trial.F90:7
  dSdpi   float64    (Lx, Ly, Lt, 3)                  gforce.F90:6
  ps      float32    (Lx+2, Ly+2, Lt+2, 2)            dum1.F90:6
  shifts  complex128 (Ls, Lx, Ly, Lt, 4, ndiag)       multishift_module.F90:29
"""
import ctypes as C
import os

import numpy as np

from . import _lib

SHAMIR, WILSON = 0, 1
NATURAL, EVEN_ODD = 0, 1
FP64, FP32_REF, MIXED_FP32, MIXED_BF16 = 0, 1, 2, 3


class TrajResult(C.Structure):
    _fields_ = [("h0", C.c_double), ("h1", C.c_double), ("dh", C.c_double), ("ds", C.c_double),
                ("s0", C.c_double), ("s1", C.c_double), ("accepted", C.c_int), ("steps", C.c_int),
                ("y", C.c_float)]


def read_remez_file(path, maxidx):
    """remez_common_subroutines.F90:20-35: returns two dicts-of-arrays pieces
    (anumA, adenA, anumB, adenB) from a text file: a0 then `a_i, s_i` lines, twice."""
    vals = []
    with open(path) as f:
        for line in f:
            line = line.replace(",", " ").split()
            if line:
                vals.append([float(v) for v in line])
    out = []
    pos = 0
    for _ in range(2):
        a0 = vals[pos][0]
        pairs = vals[pos + 1:pos + 1 + maxidx]
        pos += 1 + maxidx
        out.append((np.array([a0] + [p[0] for p in pairs]), np.array([p[1] for p in pairs])))
    (anA, adA), (anB, adB) = out
    return anA, adA, anB, adB


def remez_set(path2, path4, n):
    """The remez module arrays from the files `remez2` and `remez4` (dwf3d_lib.F90:205-209)."""
    a2, d2, b2, e2 = read_remez_file(path2, n)
    a4, d4, b4, e4 = read_remez_file(path4, n)
    return dict(anum2=a2, aden2=d2, bnum2=b2, bden2=e2, anum4=a4, aden4=d4, bnum4=b4, bden4=e4)


CON_SERIAL, CON_MPIIO = 0, 1


def read_con(path, lx, ly, lt):
    """sread (dwf3d_lib.F90:618-667): returns (theta float32 (lx,ly,lt,3) in
    Fortran order, seed, layout) from a `con` file of either layout."""
    theta = np.zeros((lx, ly, lt, 3), np.float32, order="F")
    seed = C.c_double(0)
    fmt = C.c_int(-1)
    _check(_lib.lib().thr_read_con(os.fsencode(path), lx, ly, lt, _p(theta), C.byref(seed), C.byref(fmt)), "read_con")
    return theta, seed.value, fmt.value


def write_con(path, theta, seed, layout=CON_SERIAL):
    """swrite (dwf3d_lib.F90:669-717)."""
    theta = np.asfortranarray(theta, np.float32)
    lx, ly, lt, three = theta.shape
    assert three == 3
    _check(_lib.lib().thr_write_con(os.fsencode(path), lx, ly, lt, _p(theta), float(seed), layout), "write_con")


def readseed(path):
    """readseed (dwf3d_lib.F90:719-748): the seed in a `random_seed` file."""
    v = C.c_double(0)
    _check(_lib.lib().thr_readseed(os.fsencode(path), C.byref(v)), "readseed")
    return v.value


def saveseed(path, seed):
    """saveseed (dwf3d_lib.F90:750-767)."""
    _check(_lib.lib().thr_saveseed(os.fsencode(path), float(seed)), "saveseed")


class Pack:
    """Independent lattices of uneven sizes solved together (thr_pack_*)."""

    def __init__(self, shapes, kernel=SHAMIR, am3=1.0, device=0, layout=NATURAL):
        self._L = _lib.lib()
        self.shapes = list(shapes)
        arr = (_lib.Params * len(shapes))(*[_lib.Params(lx, ly, lt, ls, kernel, layout, 25, am3, 0.4, -1, device)
                                           for (lx, ly, lt, ls) in shapes])
        h = C.c_void_p()
        _check(self._L.thr_pack_create(len(shapes), arr, device, C.byref(h)), "thr_pack_create")
        self.h = h

    def upload(self, i, u, Phi, X):
        _check(self._L.thr_pack_upload(self.h, i, _p(u), _p(Phi), _p(X)), "pack_upload")

    def zero_x(self):
        _check(self._L.thr_pack_zero_x(self.h), "pack_zero_x")

    def congrad(self, res, am, imass, precision=FP64):
        its = np.zeros(len(self.shapes), np.int32)
        outer = C.c_int(0)
        rc = self._L.thr_pack_congrad(self.h, res, am, imass, precision, _p(its), C.byref(outer))
        if rc not in (0, 3):
            _check(rc, "pack_congrad")
        return its, outer.value

    def download(self, i):
        lx, ly, lt, ls = self.shapes[i]
        X = np.zeros((ls + 2, lx + 2, ly + 2, lt + 2, 4), np.complex128, order="F")
        _check(self._L.thr_pack_download(self.h, i, _p(X)), "pack_download")
        return X

    def close(self):
        if getattr(self, "h", None):
            self._L.thr_pack_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ThirringError(RuntimeError):
    def __init__(self, status, where):
        self.status = status
        msg = _lib.lib().thr_status_string(status).decode()
        super().__init__(f"{where}: {msg} (status {status})")


def _check(rc, where):
    if rc != 0:
        raise ThirringError(rc, where)


def _p(a):
    if a is None:
        return None
    if not (a.flags.f_contiguous or a.flags.c_contiguous):
        raise ValueError("array must be contiguous")
    return a.ctypes.data_as(C.c_void_p)


def spinor(L):
    return np.zeros((L.ls + 2, L.lx + 2, L.ly + 2, L.lt + 2, 4), np.complex128, order="F")


def links(L):
    return np.zeros((L.lx + 2, L.ly + 2, L.lt + 2, 3), np.complex128, order="F")


def field3(L, dtype=np.float64):
    return np.zeros((L.lx, L.ly, L.lt, 3), dtype, order="F")


def ps_field(L):
    return np.zeros((L.lx + 2, L.ly + 2, L.lt + 2, 2), np.float32, order="F")


def shift_out(L, ndiag=None):
    return np.zeros((L.ls, L.lx, L.ly, L.lt, 4, ndiag or L.ndiag), np.complex128, order="F")


def _need(a, shape, dtype, name):
    if a.shape != shape or a.dtype != dtype or not a.flags.f_contiguous:
        raise ValueError(f"{name}: expected Fortran-ordered {dtype} array of shape {shape}, got "
                         f"{a.dtype} {a.shape}")


def zolo_coeffs(ls, lmin=0.1, lmax=5.0):
    """coeffs(1:ls) of prepZolo (measure_OWilson.F90:169-188); host only."""
    c = np.zeros(ls)
    _check(_lib.lib().thr_zolo_coeffs(ls, lmin, lmax, _p(c)), "zolo_coeffs")
    return c


class Lattice:
    """One lattice (sizes, kernel, layout) bound to one GPU context."""

    def __init__(self, lx, ly, lt, ls, kernel=SHAMIR, layout=NATURAL, ndiag=25, am3=1.0, beta=0.4,
                 ibound=-1, device=0):
        self.lx, self.ly, self.lt, self.ls = lx, ly, lt, ls
        self.kernel, self.layout, self.ndiag = kernel, layout, ndiag
        self.am3, self.beta, self.ibound = am3, beta, ibound
        self._L = _lib.lib()
        prm = _lib.Params(lx, ly, lt, ls, kernel, layout, ndiag, am3, beta, ibound, device)
        h = C.c_void_p()
        _check(self._L.thr_create(C.byref(prm), C.byref(h)), "thr_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self._L.thr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- shapes
    @property
    def sshape(self):
        return (self.ls + 2, self.lx + 2, self.ly + 2, self.lt + 2, 4)

    @property
    def ushape(self):
        return (self.lx + 2, self.ly + 2, self.lt + 2, 3)

    def set_am3(self, am3):
        self.am3 = am3
        _check(self._L.thr_set_am3(self.h, am3), "thr_set_am3")

    def set_beta(self, beta):
        self.beta = beta
        _check(self._L.thr_set_beta(self.h, beta), "thr_set_beta")

    # ---- gauge.F90
    def coef(self, theta):
        """u = coef(theta): gauge.F90:12-43.  Also becomes the current links."""
        theta = np.asfortranarray(theta, np.float32)
        _need(theta, (self.lx, self.ly, self.lt, 3), np.float32, "theta")
        u = links(self)
        _check(self._L.thr_coef(self.h, _p(u), _p(theta)), "coef")
        return u

    def set_links(self, u):
        _need(u, self.ushape, np.complex128, "u")
        _check(self._L.thr_set_links(self.h, _p(u)), "set_links")

    # ---- dirac.F90
    def dslash(self, R, u, am, imass, out=None):
        """Phi = M R  (dirac.F90:11-27).  u=None uses the current links."""
        _need(R, self.sshape, np.complex128, "R")
        if u is not None:
            _need(u, self.ushape, np.complex128, "u")
        Phi = out if out is not None else spinor(self)
        _check(self._L.thr_dslash(self.h, _p(Phi), _p(R), _p(u), am, imass), "dslash")
        return Phi

    def dslashd(self, R, u, am, imass, out=None):
        """Phi = M^dagger R  (dirac.F90:410-431)."""
        _need(R, self.sshape, np.complex128, "R")
        if u is not None:
            _need(u, self.ushape, np.complex128, "u")
        Phi = out if out is not None else spinor(self)
        _check(self._L.thr_dslashd(self.h, _p(Phi), _p(R), _p(u), am, imass), "dslashd")
        return Phi

    # ---- device fields
    def _field(self, precision, host=None):
        f = C.c_void_p()
        _check(self._L.thr_field_create(self.h, precision, C.byref(f)), "field_create")
        if host is not None:
            _need(host, self.sshape, np.complex128, "field")
            _check(self._L.thr_field_upload(self.h, f, precision, _p(host)), "field_upload")
        return f

    def dslash_fused(self, R, aux, coef, am, imass, dag, mode, precision=FP64):
        """The solvers' fused stencil epilogues on device fields (thr_dslash_fused_dev):
        mode 0 Op R, 1 aux + coef Op R, 3 Op R + coef aux (Op = M, or M^dagger for dag).
        Returns (out as a halo'd spinor, |out|^2)."""
        fs = [self._field(precision, R), self._field(precision)]
        try:
            if aux is not None:
                fs.append(self._field(precision, aux))
            n2 = C.c_double(0)
            _check(self._L.thr_dslash_fused_dev(self.h, fs[1], fs[0], fs[2] if aux is not None else None, coef,
                                                 precision, am, imass, int(dag), mode, C.byref(n2)), "dslash_fused")
            out = spinor(self)
            _check(self._L.thr_field_download(self.h, _p(out), fs[1], precision), "field_download")
            return out, n2.value
        finally:
            for f in fs:
                self._L.thr_field_destroy(self.h, f)

    def shift_residuals(self, Phi, shifts, aden, am, imass):
        """|Phi - (M^dagger M + aden[k]) x_k|^2 in FP64 for the shifted solutions
        shifts[..., k] ((Ls,Lx,Ly,Lt,4,n) as multishift_solver returns them), on the
        current links (thr_shift_residuals_dev)."""
        aden = np.ascontiguousarray(aden, np.float64)
        phi = self._field(FP64, Phi)
        try:
            r2 = np.zeros(len(aden))
            for k in range(len(aden)):
                xs = spinor(self)
                xs[1:-1, 1:-1, 1:-1, 1:-1, :] = shifts[..., k]
                xf = self._field(FP64, xs)
                try:
                    v = np.zeros(1)
                    _check(self._L.thr_shift_residuals_dev(self.h, phi, xf, 1, _p(aden[k:k + 1]), am, imass, _p(v)),
                           "shift_residuals")
                    r2[k] = v[0]
                finally:
                    self._L.thr_field_destroy(self.h, xf)
            return r2
        finally:
            self._L.thr_field_destroy(self.h, phi)

    # ---- measure_OWilson.F90
    def prep_zolo(self, lmin=0.1, lmax=5.0):
        """prepZolo (measure_OWilson.F90:169-188) on [lmin, lmax] for this Ls."""
        _check(self._L.thr_prep_zolo(self.h, lmin, lmax), "prep_zolo")

    def zolo(self):
        """The context's coeffs(1:Ls)."""
        c = np.zeros(self.ls)
        _check(self._L.thr_zolo_get(self.h, _p(c)), "zolo_get")
        return c

    def odslash(self, R, u, am, imass, out=None):
        """Phi = M_ov R  (odslash, measure_OWilson.F90:14-89).  u=None: current links."""
        _need(R, self.sshape, np.complex128, "R")
        if u is not None:
            _need(u, self.ushape, np.complex128, "u")
        Phi = out if out is not None else spinor(self)
        _check(self._L.thr_odslash(self.h, _p(Phi), _p(R), _p(u), am, imass), "odslash")
        return Phi

    def odslashd(self, R, u, am, imass, out=None):
        """Phi = M_ov^dagger R  (odslashd, measure_OWilson.F90:91-167)."""
        _need(R, self.sshape, np.complex128, "R")
        if u is not None:
            _need(u, self.ushape, np.complex128, "u")
        Phi = out if out is not None else spinor(self)
        _check(self._L.thr_odslashd(self.h, _p(Phi), _p(R), _p(u), am, imass), "odslashd")
        return Phi

    def congrad_o(self, Phi, res, am, imass):
        """congradO (measure_OWilson.F90:190-268) on the current links: returns
        (X, itercg, iterations); X starts from Phi."""
        _need(Phi, self.sshape, np.complex128, "Phi")
        X = spinor(self)
        it = C.c_int(0)
        nx = C.c_int(0)
        rc = self._L.thr_congrad_o(self.h, _p(Phi), _p(X), res, C.byref(it), am, imass, C.byref(nx))
        if rc not in (0, 3):
            _check(rc, "congrad_o")
        return X, it.value, nx.value

    # ---- random.f90 / site_random.f90 / gaussian.F90
    def init_random(self, seed, site=True):
        """init_random(seed): site streams (site_random.f90) or one global stream (random.f90)."""
        _check(self._L.thr_init_random(self.h, float(seed), int(site)), "init_random")

    def gauss0(self):
        ps = ps_field(self)
        _check(self._L.thr_gauss0(self.h, _p(ps)), "gauss0")
        return ps

    def gaussp(self):
        ps = ps_field(self)
        _check(self._L.thr_gaussp(self.h, _p(ps)), "gaussp")
        return ps

    def rano(self, ix=1, iy=1, it=1):
        v = C.c_float(0)
        _check(self._L.thr_rano(self.h, ix, iy, it, C.byref(v)), "rano")
        return v.value

    def meson(self, res, am, imass, nsource=5, precision=FP64):
        """meson(res, itercg, aviter, am, imass), measure_module.F90:684-1085."""
        lt = self.lt
        cpm, cmm = np.zeros(lt), np.zeros(lt)
        cpmn, cmmn = np.zeros(2 * lt), np.zeros(2 * lt)
        chim = C.c_double(0)
        it = C.c_int(0)
        av = C.c_float(0)
        _check(self._L.thr_meson(self.h, res, am, imass, nsource, precision, _p(cpm), _p(cmm), _p(cpmn), _p(cmmn),
                                 C.byref(chim), C.byref(it), C.byref(av)), "meson")
        return dict(cpm=cpm, cmm=cmm, cpmn=cpmn[0::2] + 1j * cpmn[1::2], cmmn=cmmn[0::2] + 1j * cmmn[1::2],
                    chim=chim.value, itercg=it.value, aviter=av.value)

    def fermion(self, res, am, imass, nsource=5, precision=FP64):
        """fermion(res, itercg, aviter, am, imass), measure_module.F90:1100-1376."""
        lt = self.lt
        c1, c2 = np.zeros(2 * lt), np.zeros(2 * lt)
        it = C.c_int(0)
        av = C.c_float(0)
        _check(self._L.thr_fermion(self.h, res, am, imass, nsource, precision, _p(c1), _p(c2), C.byref(it),
                                   C.byref(av)), "fermion")
        return dict(cferm1=c1[0::2] + 1j * c1[1::2], cferm2=c2[0::2] + 1j * c2[1::2], itercg=it.value,
                    aviter=av.value)

    def rranget(self):
        """rranget(seed, 1, 1, 1): the generator state written into checkpoints."""
        v = C.c_double(0)
        _check(self._L.thr_rranget(self.h, C.byref(v)), "rranget")
        return v.value

    def rng_state(self):
        """The complete generator state as bytes (resume with the same sequence)."""
        n = C.c_ulonglong(0)
        _check(self._L.thr_rng_state_bytes(self.h, C.byref(n)), "rng_state_bytes")
        buf = np.zeros(n.value, np.uint8)
        _check(self._L.thr_rng_save(self.h, _p(buf)), "rng_save")
        return buf.tobytes()

    def set_rng_state(self, state):
        buf = np.frombuffer(state, np.uint8).copy()
        _check(self._L.thr_rng_load(self.h, _p(buf)), "rng_load")

    # ---- measure_module.F90
    def congrad(self, Phi, X, res, am, imass):
        """congrad(Phi, res, itercg, am, imass, iterations): X (vector::X) in/out.
        Returns (itercg, iterations); raises on a non-finite residual.  Hitting
        niterc is reported by the return value status like the reference's notice."""
        _need(Phi, self.sshape, np.complex128, "Phi")
        _need(X, self.sshape, np.complex128, "X")
        it = C.c_int(0)
        nx = C.c_int(0)
        rc = self._L.thr_congrad(self.h, _p(Phi), _p(X), res, C.byref(it), am, imass, C.byref(nx))
        if rc not in (0, 3):
            _check(rc, "congrad")
        return it.value, nx.value

    def congrad_multi(self, Phi, X, res, am, imass, precision=FP64):
        """Batched congrad on the current links: Phi, X have a trailing rhs axis
        (Ls+2, Lx+2, Ly+2, Lt+2, 4, nrhs).  X in/out.  Returns (itercg[nrhs], outer rounds)."""
        nrhs = Phi.shape[-1]
        _need(Phi, self.sshape + (nrhs,), np.complex128, "Phi")
        _need(X, self.sshape + (nrhs,), np.complex128, "X")
        its = np.zeros(nrhs, np.int32)
        outer = C.c_int(0)
        rc = self._L.thr_congrad_multi(self.h, _p(Phi), _p(X), nrhs, res, am, imass, precision, _p(its),
                                       C.byref(outer))
        if rc not in (0, 3):
            _check(rc, "congrad_multi")
        return its, outer.value

    def measure(self, res, am, imass, kernel_meas=SHAMIR, knoise=10, precision=FP64):
        """measure(psibarpsi, res, aviter, am, imass), measure_module.F90:142-162,
        on the current links and random numbers.  Returns a dict with psibarpsi,
        susclsing, aviter (float32 values), parts (knoise x [Re p1, Im p1, Re p2,
        Im p2], the fort.100 columns) and itercg (one per solve).
        kernel_meas = 2 is measure_wilsonKDDW (the overlap operator,
        measure_OWilson.F90:646-673): res is then congradO's residual (the
        reference's params.F90 respbp = 1e-6), parts[n] = [Re pbp, Im pbp, 0, 0],
        four solves per noise and aviter 0 as in the reference."""
        per = 8 if kernel_meas == 1 else 4
        pb, sus, av = C.c_float(0), C.c_float(0), C.c_float(0)
        parts = np.zeros((knoise, 4), np.float64)
        its = np.zeros(per * knoise, np.int32)
        _check(self._L.thr_measure(self.h, kernel_meas, res, am, imass, knoise, precision, C.byref(pb), C.byref(sus),
                                   C.byref(av), _p(parts), _p(its)), "measure")
        return dict(psibarpsi=pb.value, susclsing=sus.value, aviter=av.value, parts=parts, itercg=its)

    def set_mixed(self, switch_fp32=1e-8, switch_bf16=1e-13):
        """Relative base residual at which the mixed multishift leaves FP64 (thr_set_mixed)."""
        _check(self._L.thr_set_mixed(self.h, switch_fp32, switch_bf16), "set_mixed")

    def mixed_switched_at(self):
        """Iteration at which the last mixed multishift left FP64 (0: it did not)."""
        v = C.c_int(0)
        _check(self._L.thr_mixed_switched_at(self.h, C.byref(v)), "mixed_switched_at")
        return v.value

    def set_solver(self, multishift_algo):
        """0: per-iteration shift updates (the reference's loop); 1: batched (default)."""
        _check(self._L.thr_set_solver(self.h, int(multishift_algo)), "set_solver")

    # ---- multishift_module.F90
    def multishift_solver(self, u, am, imass, aden, anum, inp, res, maxcg, sp=False):
        """Returns (output (Ls,Lx,Ly,Lt,4,ndiag), cg_return, cg_returns)."""
        _need(inp, self.sshape, np.complex128, "input")
        nq = len(aden)
        out = shift_out(self)
        ret = C.c_int(0)
        cgr = np.zeros(nq, np.int32)
        fn = self._L.thr_multishift_solver_sp if sp else self._L.thr_multishift_solver
        _check(fn(self.h, _p(u), am, imass, nq, _p(np.ascontiguousarray(aden, np.float64)),
                  _p(np.ascontiguousarray(anum, np.float64)), _p(out), _p(inp), res, maxcg, C.byref(ret), _p(cgr)),
               "multishift_solver")
        return out, ret.value, cgr

    # ---- qmrherm_module.F90
    def qmrherm(self, Phi, res, am, imass, anum, aden, iflag, use_sp=False, dSdpi=None, Phi0=None,
                max_qmr_iters=0):
        """x = qmrherm(Phi, …): returns (x, itercg, cg_returns).  dSdpi/Phi0 are
        updated in place when given (gforce::dSdpi, qmrherm_module::Phi0).
        use_sp: 0/False FP64, 1/True the reference's SP multishift, MIXED_FP32 or
        MIXED_BF16 the mixed multishift."""
        _need(Phi, self.sshape, np.complex128, "Phi")
        nq = len(aden)
        assert len(anum) == nq + 1
        x = spinor(self)
        it = C.c_int(0)
        cgr = np.zeros(nq, np.int32)
        if dSdpi is not None:
            _need(dSdpi, (self.lx, self.ly, self.lt, 3), np.float64, "dSdpi")
        if Phi0 is not None:
            _need(Phi0, self.sshape + (self.ndiag,), np.complex128, "Phi0")
        _check(self._L.thr_qmrherm(self.h, _p(Phi), _p(x), res, C.byref(it), am, imass,
                                   _p(np.ascontiguousarray(anum, np.float64)),
                                   _p(np.ascontiguousarray(aden, np.float64)), nq, iflag, int(use_sp), _p(cgr),
                                   _p(dSdpi), _p(Phi0), max_qmr_iters), "qmrherm")
        return x, it.value, cgr

    # ---- RHMC layer
    def set_remez(self, rat, ratg):
        """rat / ratg: dicts with anum2, aden2, bnum2, bden2, anum4, aden4, bnum4, bden4
        (remez.F90 with ndiag poles, remezg.F90 with ndiagg poles)."""
        keys = ("anum2", "aden2", "bnum2", "bden2", "anum4", "aden4", "bnum4", "bden4")
        self._keep = [np.ascontiguousarray(d[k], np.float64) for d in (rat, ratg) for k in keys]
        nd, ndg = len(rat["aden2"]), len(ratg["aden2"])
        args = [self.h, nd] + [_p(a) for a in self._keep[:8]] + [ndg] + [_p(a) for a in self._keep[8:]]
        _check(self._L.thr_set_remez(*args), "set_remez")

    def set_residuals(self, rescga=1e-8, rescgg=1e-6, spmd=1, max_qmr_iters=0):
        """params.F90:60-64; spmd is the guidance solves' qmrherm use_sp (0 FP64, 1 the
        reference's SP multishift, MIXED_FP32 / MIXED_BF16 the mixed multishift)."""
        _check(self._L.thr_set_residuals(self.h, rescga, rescgg, int(spmd), max_qmr_iters), "set_residuals")

    def set_action_precision(self, precision=FP64):
        """Precision of the Hamiltonian and pseudofermion solves (FP64, MIXED_FP32, MIXED_BF16)."""
        _check(self._L.thr_set_action_precision(self.h, int(precision)), "set_action_precision")

    def force(self, Phi, res1, am, imass, theta):
        """dSdpi = force(Phi, res1, am, imass): force_module.F90:9-113 (current links)."""
        _need(Phi, self.sshape, np.complex128, "Phi")
        theta = np.asfortranarray(theta, np.float32)
        dS = field3(self)
        _check(self._L.thr_force(self.h, _p(Phi), res1, am, imass, _p(theta), _p(dS)), "force")
        return dS

    def hamilton(self, Phi, res2, am, imass, theta, pp):
        """(h, hg, hp, s) = hamilton(Phi, …): dwf3d_lib.F90:511-616 (current links)."""
        _need(Phi, self.sshape, np.complex128, "Phi")
        theta = np.asfortranarray(theta, np.float32)
        pp = np.asfortranarray(pp, np.float32)
        v = [C.c_double(0) for _ in range(4)]
        _check(self._L.thr_hamilton(self.h, _p(Phi), *[C.byref(x) for x in v], res2, am, imass, _p(theta), _p(pp)),
               "hamilton")
        return tuple(x.value for x in v)

    def initialise_phi(self, am, imass):
        Phi = spinor(self)
        _check(self._L.thr_initialise_phi(self.h, _p(Phi), am, imass), "initialise_phi")
        return Phi

    def initialise_pp(self):
        pp = field3(self, np.float32)
        _check(self._L.thr_initialise_pp(self.h, _p(pp)), "initialise_pp")
        return pp

    def evolve_theta_pp(self, iterl, dt, pp, Phi, res, am, imass, theta, fixed_steps=0):
        """Leapfrog (evolution.F90:113-179): theta, pp updated in place; returns (itot, u, dSdpi)."""
        it = C.c_int(0)
        u = links(self)
        dS = field3(self)
        _check(self._L.thr_evolve_theta_pp(self.h, iterl, dt, _p(pp), _p(Phi), res, am, imass, C.byref(it),
                                           _p(theta), _p(u), _p(dS), fixed_steps), "evolve_theta_pp")
        return it.value, u, dS

    def trajectory(self, theta, iterl, dt, am, imass, fixed_steps=0):
        """One trajectory (dwf3d_lib.F90:265-323); theta updated in place if accepted."""
        r = TrajResult()
        _check(self._L.thr_trajectory(self.h, _p(theta), iterl, dt, am, imass, fixed_steps, C.byref(r)),
               "trajectory")
        return r

    def md_counters(self, reset=False):
        a = np.zeros(8)
        _check(self._L.thr_md_counters(self.h, _p(a), int(reset)), "md_counters")
        return dict(zip(("ancg", "ancgpv", "ancgf", "ancgfpv", "ancgh", "ancghpv", "ancgpf", "ancgpfpv"), a))

    # ---- derivs_module.F90
    def derivs(self, R, X2, anum, iflag, am, imass, dSdpi):
        """dSdpi += force of (R, X2): derivs_module.F90:8-26 (in place)."""
        _need(R, self.sshape, np.complex128, "R")
        _need(X2, self.sshape, np.complex128, "X2")
        _need(dSdpi, (self.lx, self.ly, self.lt, 3), np.float64, "dSdpi")
        _check(self._L.thr_derivs(self.h, _p(R), _p(X2), float(anum), iflag, am, imass, _p(dSdpi)), "derivs")
        return dSdpi
