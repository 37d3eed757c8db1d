"""Learned step-size proposal over the libucg C ABI (ucg_mlp_* in include/ucg.h).

A perceptron 11 -> 64 -> 64 -> 64 (GELU) -> 1 with FP16 weights proposes
log10 of the next Runge-Kutta step from the integrator's own recent history.
It is trained on the device by the library's own kernels on traces that the
ensemble integrator records (`Ensemble.record_traces`), and used by the
ensemble controller (`Ensemble.set_step_model`).  The embedded error estimate
still decides: a rejected proposal is shrunk by the plain RKQSm rule
(fortran/3d/src/ode45.f90:79-84).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import UcgError

NIN, NPARAM, NNORM, TRACE_LEN = _lib.UCG_MLP_NIN, _lib.UCG_MLP_NPARAM, _lib.UCG_MLP_NNORM, _lib.UCG_TRACE_LEN
_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)

# the step the label asks for: the one that would have met TARGET x the
# tolerance on the traced attempt (error ~ h^5), limited to a factor 10.  The
# plain controller (hnext = 0.7 h errmax^-0.2) aims at about 0.17 of the
# tolerance; a proposal aiming at 0.3 takes steps about 1.12x longer where its
# prediction holds, and each miss costs a rejected attempt
TARGET = 0.3


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def training_set(traces, target=TARGET):
    """(x, y) from trace records: x the 11 inputs, y = log10 h + 0.2 log10(target / errmax),
    clipped to log10 h +- 1."""
    t = np.asarray(traces, dtype=np.float64).reshape(-1, TRACE_LEN)
    x = t[:, :NIN]
    lh, le = t[:, NIN], t[:, NIN + 1]
    y = np.clip(lh + 0.2 * (np.log10(target) - le), lh - 1.0, lh + 1.0)
    keep = np.all(np.isfinite(x), axis=1) & np.isfinite(y)
    return x[keep].astype(np.float32), y[keep].astype(np.float32)


class StepModel:
    """The perceptron's weights on one device, with training and evaluation."""

    def __init__(self, device=0, seed=0):
        self.lib = _lib.load()
        self.mlp = ctypes.c_void_p()
        st = self.lib.ucg_mlp_create(ctypes.byref(self.mlp), device, seed)
        if st:
            raise UcgError(st, f"ucg_mlp_create: {self.lib.ucg_strerror(st).decode()}")

    def close(self):
        if self.mlp:
            self.lib.ucg_mlp_destroy(self.mlp)
            self.mlp = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st:
            msg = self.lib.ucg_mlp_last_error(self.mlp).decode() or self.lib.ucg_strerror(st).decode()
            raise UcgError(st, f"{what}: {msg}")

    def set_params(self, params=None, norm=None):
        p = _f(params) if params is not None else None
        n = _f(norm) if norm is not None else None
        self._check(self.lib.ucg_mlp_set_params(self.mlp, p.ctypes.data_as(_fp) if p is not None else None,
                                                n.ctypes.data_as(_fp) if n is not None else None), "set_params")

    def get_params(self):
        p, n = np.empty(NPARAM, np.float32), np.empty(NNORM, np.float32)
        self._check(self.lib.ucg_mlp_get_params(self.mlp, p.ctypes.data_as(_fp), n.ctypes.data_as(_fp)),
                    "get_params")
        return p, n

    def set_data(self, x, y, standardise=True):
        x, y = _f(x).reshape(-1, NIN), _f(y).ravel()
        self._check(self.lib.ucg_mlp_set_data(self.mlp, x.ctypes.data_as(_fp), y.ctypes.data_as(_fp), len(y),
                                              1 if standardise else 0), "set_data")
        self.n = len(y)

    def gradient(self, offset=0, count=None):
        count = self.n - offset if count is None else count
        g = np.empty(NPARAM, np.float32)
        loss = ctypes.c_double()
        self._check(self.lib.ucg_mlp_gradient(self.mlp, offset, count, g.ctypes.data_as(_fp), ctypes.byref(loss)),
                    "gradient")
        return loss.value, g

    def train(self, epochs=10, batch=4096, lr=1e-3, seed=0):
        losses = np.empty(epochs, np.float32)
        self._check(self.lib.ucg_mlp_train(self.mlp, epochs, batch, lr, seed, losses.ctypes.data_as(_fp)), "train")
        return losses

    def predict(self, x):
        x = _f(x).reshape(-1, NIN)
        y = np.empty(len(x), np.float32)
        self._check(self.lib.ucg_mlp_predict(self.mlp, x.ctypes.data_as(_fp), len(x), y.ctypes.data_as(_fp)),
                    "predict")
        return y
