"""Host-side mirror of the reference's 3-D rate-state / viscous-cycles drivers
over the libucg C ABI.

Names and argument meanings follow the reference:
  buildG        fortran/3d/src/greens.f90:73           -> ucg_assemble
  initStateVector fortran/3d/src/ratestate.f90:548     -> ucg_init_state
  odefun        fortran/3d/src/ratestate.f90:624       -> ucg_odefun
  RKQSm         fortran/3d/src/ode45.f90:51            -> ucg_rkqs
  main loop     fortran/3d/src/ratestate.f90:307-326   -> ucg_step / ucg_run
Errors: every non-zero status raises UcgError; the reference's "stepsize
underflow in RKQS" + STOP 1 becomes UcgError with status UCG_E_STEP_UNDERFLOW.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import UcgError

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


class Simulation:
    """One B200 context: geometry, Green's functions, state and integrator."""

    def __init__(self, mu, lam, driver="ratestate", device=0):
        self.lib = _lib.load()
        self.ctx = ctypes.c_void_p()
        drv = _lib.UCG_DRIVER_VISCOUSCYCLES if driver == "viscouscycles" else _lib.UCG_DRIVER_RATESTATE
        st = self.lib.ucg_create(ctypes.byref(self.ctx), device, float(mu), float(lam), drv)
        if st:
            raise UcgError(st, f"ucg_create: {self.lib.ucg_strerror(st).decode()}")
        self.mu, self.lam, self.driver = mu, lam, driver
        self.nr = self.nt = self.nv = 0

    @classmethod
    def adopt(cls, ctx, mu, lam, driver, nr=0, nt=0, nv=0):
        """Wrap a context created elsewhere through the C ABI (ucg_deck_create)."""
        self = cls.__new__(cls)
        self.lib = _lib.load()
        self.ctx = ctx
        self.mu, self.lam, self.driver = mu, lam, driver
        self.nr, self.nt, self.nv = nr, nt, nv
        return self

    def close(self):
        if self.ctx:
            self.lib.ucg_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st, what):
        if st:
            msg = self.lib.ucg_last_error(self.ctx).decode() or self.lib.ucg_strerror(st).decode()
            raise UcgError(st, f"{what}: {msg}")

    # ---- geometry -----------------------------------------------------------
    def set_rectangles(self, x, L, W, strike, dip):
        """x: (n, 3) upper-left corners (north, east, down); angles in radians."""
        x, L, W, strike, dip = (_d(a) for a in (x, L, W, strike, dip))
        self.nr = len(L)
        self._check(self.lib.ucg_set_rectangles(self.ctx, self.nr, _p(x), _p(L), _p(W), _p(strike),
                                                _p(dip)), "set_rectangles")

    def set_triangles(self, i1, i2, i3, v):
        """1-based vertex ids, v: (nve, 3) vertices (north, east, down)."""
        i1, i2, i3 = (np.ascontiguousarray(a, dtype=np.int32) for a in (i1, i2, i3))
        v = _d(v)
        self.nt = len(i1)
        self._check(self.lib.ucg_set_triangles(self.ctx, self.nt, _p(i1, _ip), _p(i2, _ip), _p(i3, _ip),
                                               len(v), _p(v)), "set_triangles")

    def set_volumes(self, x, L, T, W, strike):
        x, L, T, W, strike = (_d(a) for a in (x, L, T, W, strike))
        self.nv = len(L)
        self._check(self.lib.ucg_set_volumes(self.ctx, self.nv, _p(x), _p(L), _p(T), _p(W), _p(strike)),
                    "set_volumes")

    # ---- constitutive parameters ---------------------------------------------
    def set_friction(self, Vpl, rake, mu0, sig, a, b, L, Vo, damping):
        arrs = [_d(q) for q in (Vpl, rake, mu0, sig, a, b, L, Vo, damping)]
        self._check(self.lib.ucg_set_friction(self.ctx, *[_p(q) for q in arrs]), "set_friction")

    def set_rheology(self, e_bg, gammadot0m, npowerm, nonlinear_maxwell=True):
        e, g, p = _d(e_bg), _d(gammadot0m), _d(npowerm)
        self._check(self.lib.ucg_set_rheology(self.ctx, _p(e), _p(g), _p(p), int(nonlinear_maxwell)),
                    "set_rheology")

    # ---- Green's functions ---------------------------------------------------
    def buildG(self, okada_mode=_lib.UCG_OKADA_FP64):
        self._check(self.lib.ucg_assemble(self.ctx, okada_mode), "buildG")

    def build_hmatrix(self, okada_mode=_lib.UCG_OKADA_FP64, eta=2.0, eps=1.0e-6, leaf=32):
        """Hierarchical approximation of K (one patch family): clusters of `leaf`
        patches, admissibility max(diam) <= eta dist, ACA to relative accuracy eps."""
        self._check(self.lib.ucg_build_hmatrix(self.ctx, okada_mode, float(eta), float(eps), int(leaf)),
                    "build_hmatrix")

    def hmatrix_info(self):
        nd, nl, b, r, ms = ctypes.c_long(), ctypes.c_long(), ctypes.c_long(), ctypes.c_int(), ctypes.c_double()
        self._check(self.lib.ucg_hmatrix_info(self.ctx, ctypes.byref(nd), ctypes.byref(nl), ctypes.byref(b),
                                              ctypes.byref(r), ctypes.byref(ms)), "hmatrix_info")
        n, m = self.dims
        return dict(n_dense=nd.value, n_lowrank=nl.value, bytes=b.value, max_rank=r.value, build_ms=ms.value,
                    dense_bytes=8 * n * m, compression=8.0 * n * m / max(b.value, 1))

    def hmatrix_matvec(self, x):
        n, m = self.dims
        x = _d(x)
        y = np.empty(m)
        self._check(self.lib.ucg_hmatrix_matvec(self.ctx, _p(x), _p(y)), "hmatrix_matvec")
        return y

    def hmatrix_profile(self, reps=20):
        ms = ctypes.c_double()
        self._check(self.lib.ucg_hmatrix_profile(self.ctx, reps, ctypes.byref(ms)), "hmatrix_profile")
        return ms.value

    def assembly_times(self):
        """Device ms of the last buildG per source family: (rectangles, triangles, volumes)."""
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.ucg_assembly_times(self.ctx, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
                    "assembly_times")
        return a.value, b.value, c.value

    @property
    def dims(self):
        n = ctypes.c_long()
        m = ctypes.c_long()
        self._check(self.lib.ucg_dims(self.ctx, ctypes.byref(n), ctypes.byref(m)), "dims")
        return n.value, m.value

    def copy_G(self, k0=0, k1=None):
        """Columns [k0, k1) of the reference G(n,m), returned as a (k1-k0, n)
        array whose row r is column k0+r (one receiver force DOF)."""
        n, m = self.dims
        k1 = m if k1 is None else k1
        out = np.empty((k1 - k0, n))
        self._check(self.lib.ucg_copy_G(self.ctx, _p(out), n, k0, k1), "copy_G")
        return out

    def set_precision(self, precision):
        p = {"fp64": _lib.UCG_PREC_FP64, "split_bf16": _lib.UCG_PREC_SPLIT_BF16,
             "split_pair": _lib.UCG_PREC_SPLIT_PAIR}.get(precision, precision)
        self._check(self.lib.ucg_set_precision(self.ctx, p), "set_precision")

    def keep_fp64(self, keep):
        self._check(self.lib.ucg_keep_fp64(self.ctx, int(keep)), "keep_fp64")

    # ---- state and integration ----------------------------------------------
    @property
    def state_len(self):
        return self.lib.ucg_state_len(self.ctx)

    def initStateVector(self, nGm=None, nQm=None, nRm=None, To=None):
        y = np.zeros(self.state_len)
        args = [None if a is None else _d(a) for a in (nGm, nQm, nRm, To)]
        ptrs = [None if a is None else _p(a) for a in args]
        self._check(self.lib.ucg_init_state(self.ctx, _p(y), *ptrs), "initStateVector")
        return y

    def odefun(self, y, t=0.0):
        """Returns (dydt, vmax)."""
        y = _d(y)
        dydt = np.empty(self.state_len)
        vmax = ctypes.c_double()
        self._check(self.lib.ucg_odefun(self.ctx, t, _p(y), _p(dydt), ctypes.byref(vmax)), "odefun")
        return dydt, vmax.value

    def set_tolerance(self, epsilon, maximum_step=1.7976931348623158e308):
        self._check(self.lib.ucg_set_tolerance(self.ctx, epsilon, maximum_step), "set_tolerance")

    def RKQSm(self, t, y, dydt, yscal, htry):
        """One RKQSm call.  Returns (t_new, y_new, hdid, hnext, n_rejected)."""
        tt = ctypes.c_double(t)
        y = _d(y).copy()
        hdid = ctypes.c_double()
        hnext = ctypes.c_double()
        nrej = ctypes.c_long()
        self._check(self.lib.ucg_rkqs(self.ctx, ctypes.byref(tt), _p(y), _p(_d(dydt)), _p(_d(yscal)), htry,
                                      ctypes.byref(hdid), ctypes.byref(hnext), ctypes.byref(nrej)), "RKQSm")
        return tt.value, y, hdid.value, hnext.value, nrej.value

    def step(self, time, y, dt_next):
        """One main-loop iteration with host arrays.
        Returns (time, y, dydt_at_start, dt_next, dt_done, n_rejected)."""
        tm = ctypes.c_double(time)
        y = _d(y).copy()
        dydt = np.empty_like(y)
        dn = ctypes.c_double(dt_next)
        dd = ctypes.c_double()
        nrej = ctypes.c_long()
        self._check(self.lib.ucg_step(self.ctx, ctypes.byref(tm), _p(y), _p(dydt), ctypes.byref(dn),
                                      ctypes.byref(dd), ctypes.byref(nrej)), "step")
        return tm.value, y, dydt, dn.value, dd.value, nrej.value

    def set_state(self, y, time=0.0, dt_next=1.0e-3):
        self._check(self.lib.ucg_set_state(self.ctx, _p(_d(y)), time, dt_next), "set_state")

    def get_state(self):
        y = np.empty(self.state_len)
        t = ctypes.c_double()
        dn = ctypes.c_double()
        acc = ctypes.c_long()
        rej = ctypes.c_long()
        self._check(self.lib.ucg_get_state(self.ctx, _p(y), ctypes.byref(t), ctypes.byref(dn),
                                           ctypes.byref(acc), ctypes.byref(rej)), "get_state")
        return y, t.value, dn.value, acc.value, rej.value

    def run(self, t_end, max_steps):
        steps = ctypes.c_long()
        self._check(self.lib.ucg_run(self.ctx, t_end, max_steps, ctypes.byref(steps)), "run")
        return steps.value

    def set_observation_points(self, x):
        """Observation points (nobs, 3): north, east, down."""
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
        self._check(self.lib.ucg_set_observation_points(self.ctx, len(x), _p(x)), "set_observation_points")

    def buildO(self, okada_mode=_lib.UCG_OKADA_FP64):
        """Assemble the observation-point displacement kernels on the device (buildO)."""
        self._check(self.lib.ucg_build_O(self.ctx, okada_mode), "build_O")

    def observation_info(self):
        nobs, per, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self._check(self.lib.ucg_observation_info(self.ctx, ctypes.byref(nobs), ctypes.byref(per), ctypes.byref(ms)),
                    "observation_info")
        return dict(nobs=nobs.value, per_point=per.value, build_ms=ms.value)

    def copy_O(self):
        """O as a (3 nobs, n) array: row 3k + c is component c (north, east,
        down) at point k, column j the unit source DOF j of K."""
        n, _ = self.dims
        out = np.empty((3 * self.observation_info()["nobs"], n))
        self._check(self.lib.ucg_copy_O(self.ctx, _p(out)), "copy_O")
        return out

    def displacements(self, y):
        """(total, faulting, flow) displacements, each (nobs, 3), for state y."""
        y = np.ascontiguousarray(y, dtype=np.float64)
        k = self.observation_info()["nobs"]
        d, f, l = (np.empty((k, 3)) for _ in range(3))
        self._check(self.lib.ucg_displacements(self.ctx, _p(y), _p(d), _p(f), _p(l)), "displacements")
        return d, f, l

    def _pert(self, slip=None, strain=None):
        n, _ = self.dims
        u = np.zeros(n)
        np_ = self.nr + self.nt
        if slip is not None:
            u[: 2 * np_] = np.asarray(slip, dtype=np.float64).ravel()
        if strain is not None:
            u[2 * np_:] = np.asarray(strain, dtype=np.float64).ravel()
        return u

    def add_event(self, time, slip=None, strain=None):
        """Coseismic perturbation at `time`: slip (npatch, 2) strike/dip increments
        and strain (nvol, 6) eigenstrain increments; applied by run()."""
        u = self._pert(slip, strain)
        self._check(self.lib.ucg_add_event(self.ctx, float(time), _p(u)), "add_event")

    def clear_events(self):
        self._check(self.lib.ucg_clear_events(self.ctx), "clear_events")

    def apply_perturbation(self, slip=None, strain=None):
        u = self._pert(slip, strain)
        self._check(self.lib.ucg_apply_perturbation(self.ctx, _p(u)), "apply_perturbation")

    def record(self, every=1, elements=(), capacity=100000):
        """Record every `every`-th accepted step on the device (export / exportPoints);
        capacity 0 stops."""
        el = np.ascontiguousarray(elements, dtype=np.int32)
        self._check(self.lib.ucg_record(self.ctx, every, el.ctypes.data_as(_ip) if len(el) else None, len(el),
                                        capacity), "record")
        self._rec_elem = el

    def records(self, max_records=1 << 20):
        """Drained records as a dict of arrays: time, dt_done, vmax, step,
        state (n, nelem, 12), rate (n, nelem, 12), displacement (n, nobs, 3)
        (with volumes also displacement_fault and displacement_flow); and the
        number of records lost to the ring's overrun."""
        L = self.lib.ucg_record_len(self.ctx)
        buf = np.empty((max_records, L))
        n, lost = ctypes.c_long(), ctypes.c_long()
        self._check(self.lib.ucg_records(self.ctx, _p(buf), max_records, ctypes.byref(n), ctypes.byref(lost)),
                    "records")
        b = buf[:n.value]
        ne = len(getattr(self, "_rec_elem", ()))
        per = self.observation_info()["per_point"]
        nobs = (L - 4 - 24 * ne) // per
        ev = b[:, 4:4 + 24 * ne].reshape(len(b), ne, 24)
        dsp = b[:, 4 + 24 * ne:].reshape(len(b), nobs, per)
        out = dict(time=b[:, 0], dt_done=b[:, 1], vmax=b[:, 2], step=b[:, 3].astype(np.int64),
                   state=ev[:, :, :12], rate=ev[:, :, 12:], displacement=dsp[:, :, :3], lost=lost.value)
        if per == 9:
            out["displacement_fault"] = dsp[:, :, 3:6]
            out["displacement_flow"] = dsp[:, :, 6:9]
        return out

    @property
    def launch_count(self):
        return self.lib.ucg_launch_count(self.ctx)

    @property
    def stream(self):
        """The context's cudaStream_t as an integer handle."""
        return self.lib.ucg_stream(self.ctx)

    def test_wait_timeout(self, wait_ns=0, hold=False):
        """Fault injection for tests (ucg_test_wait_timeout): with hold the traction
        product's first CTA issues no copies and its consumers give up after
        wait_ns; (0, False) restores normal operation."""
        self._check(self.lib.ucg_test_wait_timeout(self.ctx, int(wait_ns), int(bool(hold))), "test_wait_timeout")

    def profile_traction(self, reps=10):
        """Mean device milliseconds of one traction-product launch."""
        ms = ctypes.c_double()
        self._check(self.lib.ucg_profile_traction(self.ctx, reps, ctypes.byref(ms)), "profile_traction")
        return ms.value
