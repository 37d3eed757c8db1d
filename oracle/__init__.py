"""ctypes bindings of the CPU oracle (liboracle.so) and of the reference's own
Nikkhoo-Walter C routine (oracle/_ref/libnw15ref.so, built from the reference
sources when they are present).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py, never by the unicycle_b200 package.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_REF = os.path.join(_HERE, "_ref", "libnw15ref.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lp = ctypes.POINTER(ctypes.c_long)

OKADA_FP64 = 0
OKADA_REF32IO = 1


def build(ref=True):
    """Compile liboracle.so, and the reference's Nikkhoo-Walter C into _ref/ when
    the environment variable UCG_REFERENCE_SRC names the reference's
    fortran/3d/src directory (there is no default location)."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    src = os.environ.get("UCG_REFERENCE_SRC")
    if not ref:
        return
    if not src:
        if not os.path.exists(_REF):
            print("oracle.build: UCG_REFERENCE_SRC is unset; the reference's own C is not compiled "
                  "(tests that need it use the committed fixtures or skip)", file=sys.stderr)
        return
    if os.path.isdir(src):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF_SRC={src}"], check=True)
    else:
        print(f"oracle.build: UCG_REFERENCE_SRC={src} is not a directory", file=sys.stderr)


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


class _Mesh(ctypes.Structure):
    _fields_ = [("nr", ctypes.c_int), ("nt", ctypes.c_int), ("nv", ctypes.c_int),
                ("rx", _dp), ("rL", _dp), ("rW", _dp), ("rstrike", _dp), ("rdip", _dp),
                ("rsv", _dp), ("rdv", _dp), ("rnv", _dp), ("rxc", _dp),
                ("nve", ctypes.c_int), ("tv", _dp), ("ti1", _ip), ("ti2", _ip), ("ti3", _ip),
                ("tsv", _dp), ("tdv", _dp), ("tnv", _dp), ("txc", _dp),
                ("vx", _dp), ("vL", _dp), ("vT", _dp), ("vW", _dp), ("vstrike", _dp),
                ("vsv", _dp), ("vdv", _dp), ("vnv", _dp), ("vxc", _dp),
                ("mu", ctypes.c_double), ("lam", ctypes.c_double),
                ("okada_mode", ctypes.c_int)]


class _Model(ctypes.Structure):
    _fields_ = [("np", ctypes.c_int), ("nvol", ctypes.c_int),
                ("Vpl", _dp), ("rake", _dp), ("mu0", _dp), ("sig", _dp), ("a", _dp),
                ("b", _dp), ("L", _dp), ("Vo", _dp), ("damping", _dp),
                ("ebg", _dp), ("gammadot0m", _dp), ("npowerm", _dp),
                ("nGm", _dp), ("nQm", _dp), ("nRm", _dp), ("To", _dp),
                ("nonlinear_maxwell", ctypes.c_int), ("viscous", ctypes.c_int),
                ("G", _dp)]


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build(ref=False)
        L = ctypes.CDLL(_LIB)
        L.orc_dc3d.restype = ctypes.c_int
        L.orc_dc3d.argtypes = [ctypes.c_int] + [ctypes.c_double] * 13 + [_dp]
        L.orc_okada_stress.argtypes = [ctypes.c_int] + [ctypes.c_double] * 15 + [_dp]
        L.orc_nw15_stress.argtypes = [ctypes.c_double] * 3 + [_dp] * 3 + [ctypes.c_double] * 5 + [_dp]
        L.orc_bml17_stress.argtypes = [ctypes.c_double] * 10 + [_dp, ctypes.c_double, ctypes.c_double, _dp]
        L.orc_bml17_stress_mindlin.argtypes = [ctypes.c_double] * 10 + [_dp, ctypes.c_double, ctypes.c_double, _dp]
        L.orc_cuboid_grad_mindlin.argtypes = [ctypes.c_double] * 7 + [_dp, ctypes.c_double, ctypes.c_double, _dp]
        L.orc_mindlin.argtypes = [ctypes.c_double] * 6 + [_dp]
        L.orc_okada_frames.argtypes = [ctypes.c_int] + [_dp] * 9
        L.orc_tri_frames.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _ip, _ip, _ip] + [_dp] * 4
        L.orc_vol_frames.argtypes = [ctypes.c_int] + [_dp] * 8
        L.orc_g_rows.restype = ctypes.c_long
        L.orc_g_cols.restype = ctypes.c_long
        L.orc_g_rows.argtypes = [ctypes.POINTER(_Mesh)]
        L.orc_g_cols.argtypes = [ctypes.POINTER(_Mesh)]
        L.orc_build_g.argtypes = [ctypes.POINTER(_Mesh), ctypes.c_long, ctypes.c_long, _dp]
        L.orc_build_g_omp.argtypes = [ctypes.POINTER(_Mesh), ctypes.c_long, ctypes.c_long, _dp, ctypes.c_int]
        L.orc_dgemv_t.argtypes = [ctypes.c_long, ctypes.c_long, _dp, _dp, _dp, ctypes.c_int]
        L.orc_state_len.restype = ctypes.c_long
        L.orc_state_len.argtypes = [ctypes.POINTER(_Model)]
        L.orc_work_len.restype = ctypes.c_long
        L.orc_work_len.argtypes = [ctypes.POINTER(_Model)]
        L.orc_init_state.argtypes = [ctypes.POINTER(_Model), _dp]
        L.orc_odefun.argtypes = [ctypes.POINTER(_Model), _dp, _dp, _dp, _dp]
        L.orc_rkck.argtypes = [ctypes.POINTER(_Model), _dp, _dp, ctypes.c_double, _dp, _dp, _dp]
        L.orc_rkqs.restype = ctypes.c_int
        L.orc_rkqs.argtypes = [ctypes.POINTER(_Model), _dp, _dp, _dp, _dp, ctypes.c_double,
                               ctypes.c_double, ctypes.c_double, _dp, _dp, _lp, _dp]
        L.orc_step.restype = ctypes.c_int
        L.orc_step.argtypes = [ctypes.POINTER(_Model), _dp, _dp, _dp, _dp, ctypes.c_double,
                               ctypes.c_double, _dp, _lp, _dp]
        L.orc_okada_disp.argtypes = [ctypes.c_int] + [ctypes.c_double] * 15 + [_dp]
        L.orc_nw15_disp.argtypes = [ctypes.c_double] * 3 + [_dp] * 3 + [ctypes.c_double] * 5 + [_dp]
        L.orc_bml17_disp_ned.argtypes = [ctypes.c_double] * 10 + [_dp, ctypes.c_double, ctypes.c_double, _dp]
        L.orc_build_o.argtypes = [ctypes.POINTER(_Mesh), ctypes.c_int, _dp, _dp]
        _fp = ctypes.POINTER(ctypes.c_float)
        L.orc_mlp_nparam.restype = ctypes.c_int
        L.orc_mlp_loss_grad.argtypes = [_fp, _fp, _fp, _fp, ctypes.c_long, ctypes.c_int, _dp, _dp]
        L.orc_mlp_predict.argtypes = [_fp, _fp, _fp, ctypes.c_long, ctypes.c_int, _dp]
        _lib = L
    return _lib


def ref_lib():
    """The reference's straininhalfspace_ compiled from its own sources, or None."""
    global _ref
    if _ref is None and os.path.exists(_REF):
        R = ctypes.CDLL(_REF)
        R.straininhalfspace_.argtypes = [_dp, _dp] + [ctypes.c_double] * 3 + [_dp] * 3 + [ctypes.c_double] * 5
        R.straininhalfspace_.restype = None
        _ref = R
    return _ref


def _d(x):
    return np.ascontiguousarray(x, dtype=np.float64)


def dc3d(mode, alpha, x, y, z, depth, dip_deg, al1, al2, aw1, aw2, d1, d2, d3):
    u = np.zeros(12)
    ret = lib().orc_dc3d(mode, alpha, x, y, z, depth, dip_deg, al1, al2, aw1, aw2, d1, d2, d3, _ptr(u))
    return ret, u


def okada_stress(mode, x, q, L, W, strike, dip, s, d, t, G, lam):
    sig = np.zeros(6)
    lib().orc_okada_stress(mode, x[0], x[1], x[2], q[0], q[1], q[2], L, W, strike, dip,
                           s, d, t, G, lam, _ptr(sig))
    return sig


def nw15_stress(x, P1, P2, P3, s, d, t, G, lam):
    sig = np.zeros(6)
    lib().orc_nw15_stress(x[0], x[1], x[2], _ptr(_d(P1)), _ptr(_d(P2)), _ptr(_d(P3)),
                          s, d, t, G, lam, _ptr(sig))
    return sig


def nw15_stress_ref(x, P1, P2, P3, s, d, t, G, lam):
    """computeStressNikkhoo15 (nikkhoo15.f90:120-163) around the reference C."""
    R = ref_lib()
    if R is None:
        return None
    Q = [_d([P[1], P[0], -P[2]]) for P in (P1, P2, P3)]
    st = np.zeros(6)
    e = np.zeros(6)
    R.straininhalfspace_(_ptr(st), _ptr(e), x[1], x[0], -x[2], _ptr(Q[0]), _ptr(Q[1]),
                         _ptr(Q[2]), s, -d, t, G, lam)
    return np.array([st[3], st[1], -st[4], st[0], -st[2], st[5]])


def bml17_stress(x, q, L, T, W, theta, eps, G, nu):
    sig = np.zeros(6)
    lib().orc_bml17_stress(x[0], x[1], x[2], q[0], q[1], q[2], L, T, W, theta,
                           _ptr(_d(eps)), G, nu, _ptr(sig))
    return sig


def bml17_stress_mindlin(x, q, L, T, W, theta, eps, G, nu):
    """The cuboid's stress by Mindlin's point force integrated over its faces
    (oracle/mindlin.cc), independent of the Barbot et al. closed forms."""
    sig = np.zeros(6)
    lib().orc_bml17_stress_mindlin(x[0], x[1], x[2], q[0], q[1], q[2], L, T, W, theta,
                                   _ptr(_d(eps)), G, nu, _ptr(sig))
    return sig


def set_dgemv_threads(threads):
    """odefun's DGEMV over `threads` threads in a plain summation order (timing
    the CPU baseline); 0 restores the fixed order the parity tests use."""
    lib().orc_set_dgemv_threads(int(threads))


def set_volume_route(route):
    """Strain-volume sources in Mesh.build_g: 0 the closed forms (default), 1
    Mindlin's point force over the cuboid's faces (independent route)."""
    lib().orc_set_volume_route(int(route))


def mindlin(x, y, z, c, G, nu):
    """Mindlin's half-space Green's function: u[i, j] at (x, y, z) from a unit
    force along j at (0, 0, c)."""
    u = np.zeros(9)
    lib().orc_mindlin(x, y, z, c, G, nu, _ptr(u))
    return u.reshape(3, 3)


class Mesh:
    """Geometry for orc_build_g.  Arrays follow the reference's (3, n) Fortran
    layout, stored here as (n, 3) C-contiguous."""

    def __init__(self, mu, lam, rect=None, tri=None, vol=None, okada_mode=OKADA_FP64):
        self._keep = []
        m = _Mesh()
        m.mu, m.lam, m.okada_mode = mu, lam, okada_mode
        L = lib()
        if rect is not None:
            x, Lr, Wr, st, dp = (_d(a) for a in rect)
            n = len(Lr)
            sv, dv, nv, xc = (np.zeros((n, 3)) for _ in range(4))
            L.orc_okada_frames(n, _ptr(x), _ptr(Lr), _ptr(Wr), _ptr(st), _ptr(dp),
                               _ptr(sv), _ptr(dv), _ptr(nv), _ptr(xc))
            self._keep += [x, Lr, Wr, st, dp, sv, dv, nv, xc]
            m.nr = n
            m.rx, m.rL, m.rW, m.rstrike, m.rdip = (_ptr(a) for a in (x, Lr, Wr, st, dp))
            m.rsv, m.rdv, m.rnv, m.rxc = (_ptr(a) for a in (sv, dv, nv, xc))
            self.rect_frames = (sv, dv, nv, xc)
        if tri is not None:
            v, i1, i2, i3 = tri
            v = _d(v)
            i1, i2, i3 = (np.ascontiguousarray(a, dtype=np.int32) for a in (i1, i2, i3))
            n = len(i1)
            sv, dv, nv, xc = (np.zeros((n, 3)) for _ in range(4))
            L.orc_tri_frames(n, len(v), _ptr(v), _ptr(i1, _ip), _ptr(i2, _ip), _ptr(i3, _ip),
                             _ptr(sv), _ptr(dv), _ptr(nv), _ptr(xc))
            self._keep += [v, i1, i2, i3, sv, dv, nv, xc]
            m.nt, m.nve = n, len(v)
            m.tv, m.ti1, m.ti2, m.ti3 = _ptr(v), _ptr(i1, _ip), _ptr(i2, _ip), _ptr(i3, _ip)
            m.tsv, m.tdv, m.tnv, m.txc = (_ptr(a) for a in (sv, dv, nv, xc))
            self.tri_frames = (sv, dv, nv, xc)
        if vol is not None:
            x, Lv, Tv, Wv, st = (_d(a) for a in vol)
            n = len(Lv)
            sv, dv, nv, xc = (np.zeros((n, 3)) for _ in range(4))
            L.orc_vol_frames(n, _ptr(x), _ptr(Lv), _ptr(Wv), _ptr(st), _ptr(sv), _ptr(dv),
                             _ptr(nv), _ptr(xc))
            self._keep += [x, Lv, Tv, Wv, st, sv, dv, nv, xc]
            m.nv = n
            m.vx, m.vL, m.vT, m.vW, m.vstrike = (_ptr(a) for a in (x, Lv, Tv, Wv, st))
            m.vsv, m.vdv, m.vnv, m.vxc = (_ptr(a) for a in (sv, dv, nv, xc))
            self.vol_frames = (sv, dv, nv, xc)
        self.m = m

    @property
    def n(self):
        return lib().orc_g_rows(ctypes.byref(self.m))

    @property
    def mcols(self):
        return lib().orc_g_cols(ctypes.byref(self.m))

    def build_o(self, xobs):
        """O (3 nobs x n, row-major): displacement (north, east, down) at the points
        for unit slip / eigenstrain on every source (greens.f90:302-462)."""
        xobs = _d(xobs).reshape(-1, 3)
        O = np.zeros((3 * len(xobs), self.n))
        lib().orc_build_o(ctypes.byref(self.m), len(xobs), _ptr(xobs), _ptr(O))
        return O

    def build_g(self, k0=0, k1=None):
        """Columns [k0,k1) of the reference G(n,m); returned as (k1-k0, n), i.e.
        row r of the result is column k0+r of G (a receiver DOF)."""
        if k1 is None:
            k1 = self.mcols
        G = np.zeros((k1 - k0, self.n))
        lib().orc_build_g(ctypes.byref(self.m), k0, k1, _ptr(G))
        return G


class Model:
    """Rate-state (+ Maxwell volume) model around a dense G (numpy, shape (m, n):
    row k is column k of the reference G)."""

    def __init__(self, G, patch, vol=None, viscous=False, nonlinear_maxwell=False):
        self._keep = []
        md = _Model()
        self.G = None if G is None else np.ascontiguousarray(G, dtype=np.float64)
        np_ = len(patch["Vpl"])
        md.np = np_
        for k in ("Vpl", "rake", "mu0", "sig", "a", "b", "L", "Vo", "damping"):
            a = _d(patch[k])
            self._keep.append(a)
            setattr(md, k, _ptr(a))
        md.nvol = 0
        if vol is not None:
            md.nvol = len(vol["gammadot0m"])
            for k in ("ebg", "gammadot0m", "npowerm", "nGm", "nQm", "nRm", "To"):
                a = _d(vol[k])
                self._keep.append(a)
                setattr(md, k, _ptr(a))
        md.viscous = int(viscous)
        md.nonlinear_maxwell = int(nonlinear_maxwell)
        md.G = _ptr(self.G) if self.G is not None else ctypes.cast(None, _dp)
        self.md = md
        self.len = lib().orc_state_len(ctypes.byref(md))
        self.work = np.zeros(lib().orc_work_len(ctypes.byref(md)) + 16)

    def init_state(self):
        y = np.zeros(self.len)
        lib().orc_init_state(ctypes.byref(self.md), _ptr(y))
        return y

    def odefun(self, y):
        y = _d(y)
        dydt = np.zeros(self.len)
        vmax = np.zeros(1)
        lib().orc_odefun(ctypes.byref(self.md), _ptr(y), _ptr(dydt), _ptr(vmax), _ptr(self.work))
        return dydt, vmax[0]

    def rkck(self, y, dydt, h):
        yout = np.zeros(self.len)
        yerr = np.zeros(self.len)
        lib().orc_rkck(ctypes.byref(self.md), _ptr(_d(y)), _ptr(_d(dydt)), h, _ptr(yout),
                       _ptr(yerr), _ptr(self.work))
        return yout, yerr

    def rkqs(self, y, dydt, yscal, htry, eps, hmax=1.7976931348623158e308):
        y = _d(y).copy()
        t = np.zeros(1)
        hdid = np.zeros(1)
        hnext = np.zeros(1)
        nrej = np.zeros(1, dtype=np.int64)
        rc = lib().orc_rkqs(ctypes.byref(self.md), _ptr(t), _ptr(y), _ptr(_d(dydt)), _ptr(_d(yscal)),
                            htry, eps, hmax, _ptr(hdid), _ptr(hnext), _ptr(nrej, _lp), _ptr(self.work))
        return rc, y, hdid[0], hnext[0], int(nrej[0])

    def step(self, time, y, dt_next, eps, hmax=1.7976931348623158e308):
        """One main-loop iteration.  Returns (rc, time, y, dydt_at_start, dt_next, dt_done, nrej)."""
        y = _d(y).copy()
        tm = np.array([time], dtype=np.float64)
        dydt = np.zeros(self.len)
        dn = np.array([dt_next], dtype=np.float64)
        dd = np.zeros(1)
        nrej = np.zeros(1, dtype=np.int64)
        rc = lib().orc_step(ctypes.byref(self.md), _ptr(tm), _ptr(y), _ptr(dydt), _ptr(dn), eps,
                            hmax, _ptr(dd), _ptr(nrej, _lp), _ptr(self.work))
        return rc, tm[0], y, dydt, dn[0], dd[0], int(nrej[0])


def build_g_omp(mesh, k0, k1, threads):
    """Columns [k0,k1) of G assembled with `threads` OpenMP threads; (k1-k0, n)."""
    G = np.zeros((k1 - k0, mesh.n))
    lib().orc_build_g_omp(ctypes.byref(mesh.m), k0, k1, _ptr(G), threads)
    return G


def dgemv_t(Gblock, v, threads):
    """t = G^T v for a block given as (m, n) rows (= reference G columns)."""
    Gblock = np.ascontiguousarray(Gblock, dtype=np.float64)
    v = _d(v)
    t = np.zeros(Gblock.shape[0])
    lib().orc_dgemv_t(Gblock.shape[1], Gblock.shape[0], _ptr(Gblock), _ptr(v), _ptr(t), threads)
    return t


def rk_overhead_seconds(cfg, reps=3):
    """Seconds of one oracle main-loop step without the matrix-vector products
    (the O(N) elementwise right-hand side, BLAS-1 stage combinations, error
    norm and control) at the config's full size."""
    import time
    md = Model(None, cfg["friction"])
    y = cfg["y0"].copy()
    t, dt = 0.0, cfg["dt0"]
    t0 = time.perf_counter()
    for _ in range(reps):
        rc, t, y, _, dt, _, _ = md.step(t, y, dt, cfg["epsilon"])
    return (time.perf_counter() - t0) / reps


def _f(x):
    return np.ascontiguousarray(x, dtype=np.float32)


def mlp_loss_grad(params, norm, X, Y, fp16=True, grad=True):
    """Mean loss and its gradient for the step-size perceptron (oracle/mlp.c)."""
    L = lib()
    params, norm, X, Y = _f(params), _f(norm), _f(X), _f(Y)
    fp = ctypes.POINTER(ctypes.c_float)
    g = np.zeros(L.orc_mlp_nparam()) if grad else None
    loss = np.zeros(1)
    L.orc_mlp_loss_grad(params.ctypes.data_as(fp), norm.ctypes.data_as(fp), X.ctypes.data_as(fp),
                        Y.ctypes.data_as(fp), len(Y), 1 if fp16 else 0,
                        g.ctypes.data_as(_dp) if grad else None, _ptr(loss))
    return loss[0], g


def mlp_predict(params, norm, X, fp16=True):
    L = lib()
    params, norm, X = _f(params), _f(norm), _f(X)
    fp = ctypes.POINTER(ctypes.c_float)
    out = np.zeros(X.shape[0])
    L.orc_mlp_predict(params.ctypes.data_as(fp), norm.ctypes.data_as(fp), X.ctypes.data_as(fp), X.shape[0],
                      1 if fp16 else 0, _ptr(out))
    return out


def nw15_disp_ref(x, P1, P2, P3, s, d, t, G, lam):
    """The reference's own dispinhalfspace_ (compiled from its sources) with the
    NED conventions of computeDisplacementNikkhoo15 (nikkhoo15.f90:324-367)."""
    R = ref_lib()
    if R is None:
        return None
    if not hasattr(R, "_disp_bound"):
        R.dispinhalfspace_.argtypes = [_dp] + [ctypes.c_double] * 3 + [_dp] * 3 + [ctypes.c_double] * 4
        R.dispinhalfspace_.restype = None
        R._disp_bound = True
    nu = lam / (lam + G) / 2.0
    q = [_d([p[1], p[0], -p[2]]) for p in (P1, P2, P3)]
    u = np.zeros(3)
    R.dispinhalfspace_(_ptr(u), x[1], x[0], -x[2], _ptr(q[0]), _ptr(q[1]), _ptr(q[2]), s, -d, t, nu)
    return np.array([u[1], u[0], -u[2]])


def nw15_disp(x, P1, P2, P3, s, d, t, G, lam):
    u = np.zeros(3)
    lib().orc_nw15_disp(x[0], x[1], x[2], _ptr(_d(P1)), _ptr(_d(P2)), _ptr(_d(P3)), s, d, t, G, lam, _ptr(u))
    return u


def okada_disp(mode, x, q, L, W, strike, dip, s, d, t, G, lam):
    u = np.zeros(3)
    lib().orc_okada_disp(mode, x[0], x[1], x[2], q[0], q[1], q[2], L, W, strike, dip, s, d, t, G, lam, _ptr(u))
    return u


def bml17_disp(x, q, L, T, W, theta, eps, G, nu):
    """Displacement (north, east, down) of a cuboid with eigenstrain eps
    (strainvolume.f90:215-991, computeDisplacementVerticalStrainVolume)."""
    u = np.zeros(3)
    lib().orc_bml17_disp_ned(x[0], x[1], x[2], q[0], q[1], q[2], L, T, W, theta, _ptr(_d(eps)), G, nu, _ptr(u))
    return u
