"""Batched ensembles over the libucg C ABI (ucg_ens_* in include/ucg.h).

Many frictional-parameter instances of one or more fault geometries march
together; the traction product of every Runge-Kutta stage is one tensor-core
contraction per geometry.  Each instance follows the reference main loop
(fortran/3d/src/ratestate.f90:307-326) with its own step size and RKQSm
decision (fortran/3d/src/ode45.f90:51-108).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import UcgError
from .simulation import _d, _p

_ip = ctypes.POINTER(ctypes.c_int)


class Ensemble:
    """Instances of fault geometries marched together on one device."""

    def __init__(self, device=0):
        self.lib = _lib.load()
        self.ens = ctypes.c_void_p()
        st = self.lib.ucg_ens_create(ctypes.byref(self.ens), device)
        if st:
            raise UcgError(st, f"ucg_ens_create: {self.lib.ucg_strerror(st).decode()}")
        self.geoms = []   # (n_patches, n_instances)

    def close(self):
        if self.ens:
            self.lib.ucg_ens_destroy(self.ens)
            self.ens = ctypes.c_void_p()

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
            msg = self.lib.ucg_ens_last_error(self.ens).decode() or self.lib.ucg_strerror(st).decode()
            raise UcgError(st, f"{what}: {msg}")

    def add_geometry(self, sim, n_instances):
        """Add the geometry of `sim` (a Simulation) with n_instances instances: its assembled
        dense K, or its hierarchical matrix when `sim` steps on it (UCG_PREC_HMATRIX after
        build_hmatrix, leaf <= 42) or holds no dense K; the hierarchical operand images are
        built here."""
        g = ctypes.c_int()
        self._check(self.lib.ucg_ens_add_geometry(self.ens, sim.ctx, int(n_instances), ctypes.byref(g)),
                    "add_geometry")
        n, m = sim.dims
        self.geoms.append((n // 2, int(n_instances), n, m))
        return g.value

    def set_friction(self, geometry, instance, Vpl, rake, mu0, sig, a, b, L, Vo, damping):
        arrs = [_d(x) for x in (Vpl, rake, mu0, sig, a, b, L, Vo, damping)]
        self._check(self.lib.ucg_ens_set_friction(self.ens, geometry, instance, *[_p(x) for x in arrs]),
                    "set_friction")

    def set_tolerance(self, epsilon, maximum_step=1.7976931348623158e308):
        self._check(self.lib.ucg_ens_set_tolerance(self.ens, epsilon, maximum_step), "set_tolerance")

    def set_state(self, geometry, instance, y, time=0.0, dt_next=1.0e-3):
        self._check(self.lib.ucg_ens_set_state(self.ens, geometry, instance, time, _p(_d(y)), dt_next),
                    "set_state")

    def get_state(self, geometry, instance):
        """Returns (y, time, dt_next, accepted, rejected, status)."""
        y = np.empty(7 * self.geoms[geometry][0])
        t, dn = ctypes.c_double(), ctypes.c_double()
        acc, rej = ctypes.c_long(), ctypes.c_long()
        st = ctypes.c_int()
        self._check(self.lib.ucg_ens_get_state(self.ens, geometry, instance, _p(y), ctypes.byref(t),
                                               ctypes.byref(dn), ctypes.byref(acc), ctypes.byref(rej),
                                               ctypes.byref(st)), "get_state")
        return y, t.value, dn.value, acc.value, rej.value, st.value

    def set_states(self, geometry, y, time, dt_next):
        """All instances of a geometry: y (n_instances, 7 n), time and dt_next (n_instances,)."""
        ninst = self.geoms[geometry][1]
        y = _d(y).reshape(ninst, -1)
        t = _d(np.broadcast_to(np.asarray(time, dtype=float), (ninst,)))
        dn = _d(np.broadcast_to(np.asarray(dt_next, dtype=float), (ninst,)))
        self._check(self.lib.ucg_ens_set_states(self.ens, geometry, _p(y), _p(t), _p(dn)), "set_states")

    def put_states(self, geometry, y):
        """Replace every instance's state (n_instances, 7 n) and keep its time, step
        size, counters and step history (ucg_ens_put_states): the states taken by
        get_states and handed back continue as the device-resident loop would."""
        ninst = self.geoms[geometry][1]
        y = _d(y).reshape(ninst, -1)
        self._check(self.lib.ucg_ens_put_states(self.ens, geometry, _p(y)), "put_states")

    def set_increment_terms(self, terms):
        """Stage increments in the anchor's three-term form (3, the default) or the
        two-term form Khi (Vhi + Vlo) (2) (ucg_ens_set_increment_terms)."""
        self._check(self.lib.ucg_ens_set_increment_terms(self.ens, int(terms)), "set_increment_terms")

    def set_hier_planes(self, planes):
        """bf16 planes of the hierarchical geometries' operand images: 3 (24 bits,
        the default) or 2 (16 bits); before the first hierarchical geometry is
        added (ucg_ens_set_hier_planes)."""
        self._check(self.lib.ucg_ens_set_hier_planes(self.ens, int(planes)), "set_hier_planes")

    def test_wait_timeout(self, wait_ns=0, hold=False):
        """Fault injection for tests (ucg_ens_test_wait_timeout): with hold the dense
        contraction's first CTA issues no copies and its MMA issuer gives up after
        wait_ns; (0, False) restores normal operation."""
        self._check(self.lib.ucg_ens_test_wait_timeout(self.ens, int(wait_ns), int(bool(hold))),
                    "test_wait_timeout")

    def get_states(self, geometry, out=None):
        """(y (n_instances, 7 n), time, dt_next, accepted, rejected, status) of all instances."""
        npatch, ninst = self.geoms[geometry][0], self.geoms[geometry][1]
        y = out if out is not None else np.empty((ninst, 7 * npatch))
        t, dn = np.empty(ninst), np.empty(ninst)
        acc, rej = np.empty(ninst, dtype=np.int64), np.empty(ninst, dtype=np.int64)
        st = np.empty(ninst, dtype=np.int32)
        lp = ctypes.POINTER(ctypes.c_long)
        self._check(self.lib.ucg_ens_get_states(self.ens, geometry, _p(y), _p(t), _p(dn), acc.ctypes.data_as(lp),
                                                rej.ctypes.data_as(lp), st.ctypes.data_as(_ip)), "get_states")
        return y, t, dn, acc, rej, st

    def plan(self, ni=64, schedule=_lib.UCG_ENS_STREAM_K, chunk=0):
        self._check(self.lib.ucg_ens_plan(self.ens, ni, schedule, chunk), "plan")

    def tune(self, reps=5):
        """Time every candidate contraction plan, install the fastest, return the report."""
        buf = ctypes.create_string_buffer(8192)
        self._check(self.lib.ucg_ens_tune(self.ens, reps, buf, len(buf)), "tune")
        return buf.value.decode()

    def use_graph(self, flag=True):
        """Attempts as one CUDA-graph launch (default) or host-launched kernels."""
        self._check(self.lib.ucg_ens_use_graph(self.ens, 1 if flag else 0), "use_graph")

    def run(self, t_end, max_attempts):
        """March every instance to t_end; returns the attempts made."""
        n = ctypes.c_long()
        self._check(self.lib.ucg_ens_run(self.ens, t_end, max_attempts, ctypes.byref(n)), "run")
        return n.value

    def matvec(self, geometry, V, terms=3):
        """T = K V through the tensor-core contraction; V: (n_instances, n) -> (n_instances, m).
        terms=3: the anchor's product (K hi and lo), terms=2: the increments' (K hi only)."""
        _, ninst, n, m = self.geoms[geometry]
        V = _d(V).reshape(ninst, n)
        T = np.empty((ninst, m))
        self._check(self.lib.ucg_ens_matvec(self.ens, geometry, _p(V), _p(T), int(terms)), "matvec")
        return T

    def set_event_threshold(self, vmax_on=1.0e-3, vmax_off=1.0e-4):
        self._check(self.lib.ucg_ens_set_event_threshold(self.ens, vmax_on, vmax_off), "set_event_threshold")

    def events(self, geometry, instance):
        """(number of events, start time of the first event or -1)."""
        ne, tf = ctypes.c_long(), ctypes.c_double()
        self._check(self.lib.ucg_ens_get_events(self.ens, geometry, instance, ctypes.byref(ne), ctypes.byref(tf)),
                    "events")
        return ne.value, tf.value

    def set_step_model(self, model):
        """Use a StepModel's proposals for every instance (None: the plain controller)."""
        self._check(self.lib.ucg_ens_set_step_model(self.ens, model.mlp if model is not None else None),
                    "set_step_model")
        self._model = model   # keep it alive while in use

    def record_traces(self, capacity):
        """Start recording step traces (capacity records); 0 stops."""
        self._check(self.lib.ucg_ens_record_traces(self.ens, int(capacity)), "record_traces")

    def traces(self):
        """The recorded traces, (n, 14) float32."""
        from .stepmodel import TRACE_LEN
        n = ctypes.c_long()
        self._check(self.lib.ucg_ens_get_traces(self.ens, None, 0, ctypes.byref(n)), "traces")
        buf = np.empty((n.value, TRACE_LEN), np.float32)
        if n.value:
            self._check(self.lib.ucg_ens_get_traces(self.ens, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                    n.value, ctypes.byref(n)), "traces")
        return buf

    def info(self):
        """dict: attempts, active, launches, accepted, rejected, time_sum, plan."""
        ta, act, la = ctypes.c_long(), ctypes.c_int(), ctypes.c_long()
        acc, rej, ts = ctypes.c_long(), ctypes.c_long(), ctypes.c_double()
        buf = ctypes.create_string_buffer(1024)
        self._check(self.lib.ucg_ens_info(self.ens, ctypes.byref(ta), ctypes.byref(act), ctypes.byref(la),
                                          ctypes.byref(acc), ctypes.byref(rej), ctypes.byref(ts), buf, len(buf)),
                    "info")
        return dict(attempts=ta.value, active=act.value, launches=la.value, accepted=acc.value,
                    rejected=rej.value, time_sum=ts.value, plan=buf.value.decode())

    @property
    def stream(self):
        """The ensemble's cudaStream_t as an integer handle."""
        return self.lib.ucg_ens_stream(self.ens)

    def profile_contract(self, reps=10):
        """Mean device ms per launch: (anchor form, increment form)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.ucg_ens_profile_contract(self.ens, reps, ctypes.byref(a), ctypes.byref(b)),
                    "profile_contract")
        return a.value, b.value
