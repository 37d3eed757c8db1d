"""Input decks of the reference's 3-D drivers (init() of
fortran/3d/src/ratestate.f90:958-1739 and viscouscycles.f90:1291-2069):
parsing through libucg (ucg_deck_*), loading into a Simulation, the whole run
(ucg_deck_run), and a writer that turns the synthetic configurations of
unicycle_b200.configs into decks of the same format."""
import ctypes
import os

import numpy as np

from . import _lib
from ._lib import UcgError
from .simulation import Simulation

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)

_DOUBLE_FIELDS = ("rect.x", "rect.length", "rect.width", "rect.strike", "rect.dip", "tri.vertices", "patch.Vpl",
                  "patch.rake", "patch.mu0", "patch.sig", "patch.a", "patch.b", "patch.L", "patch.Vo",
                  "patch.damping", "vol.x", "vol.length", "vol.width", "vol.thickness", "vol.strike", "vol.e_bg",
                  "vol.Gm", "vol.gammadot0m", "vol.npowerm", "vol.Q", "vol.R", "vol.rhoc", "vol.To", "obs.x",
                  "events.time")
_INT_FIELDS = ("tri.i1", "tri.i2", "tri.i3", "obs.state")


def _driver_code(driver):
    return _lib.UCG_DRIVER_VISCOUSCYCLES if driver == "viscouscycles" else _lib.UCG_DRIVER_RATESTATE


class Deck:
    """A parsed deck.  Deck(text) or Deck.read(path); driver "ratestate" or
    "viscouscycles" selects the section layout."""

    def __init__(self, text, driver="ratestate", _path=None):
        self.lib = _lib.load()
        self.h = ctypes.c_void_p()
        self.driver = driver
        err = ctypes.create_string_buffer(512)
        if _path is not None:
            st = self.lib.ucg_deck_read(_path.encode(), _driver_code(driver), ctypes.byref(self.h), err, 512)
        else:
            st = self.lib.ucg_deck_parse(text.encode(), _driver_code(driver), ctypes.byref(self.h), err, 512)
        if st:
            raise UcgError(st, err.value.decode() or self.lib.ucg_strerror(st).decode())

    @classmethod
    def read(cls, path, driver="ratestate"):
        return cls(None, driver, _path=os.fspath(path))

    def close(self):
        if self.h:
            self.lib.ucg_deck_free(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def info(self):
        s = _lib.DeckInfo()
        self.lib.ucg_deck_summary(self.h, ctypes.byref(s))
        d = {f: getattr(s, f) for f, _ in s._fields_}
        d["lambda"] = d.pop("lambda_")
        d["wdir"] = self.lib.ucg_deck_wdir(self.h).decode()
        d["point_names"] = [self.lib.ucg_deck_point_name(self.h, k).decode() for k in range(s.n_obs_point)]
        return d

    def get(self, field):
        """A field as a numpy array (angles in radians; indices 1-based)."""
        if field in _INT_FIELDS:
            n = self.lib.ucg_deck_get_int(self.h, field.encode(), None, 0)
            out = np.zeros(n, dtype=np.int32)
            self.lib.ucg_deck_get_int(self.h, field.encode(), out.ctypes.data_as(_ip), n)
            return out
        if field not in _DOUBLE_FIELDS:
            raise KeyError(field)
        n = self.lib.ucg_deck_get(self.h, field.encode(), None, 0)
        out = np.zeros(n)
        self.lib.ucg_deck_get(self.h, field.encode(), out.ctypes.data_as(_dp), n)
        return out

    def simulation(self, device=0):
        """A Simulation holding the deck's elements, friction, rheology and
        observation points (not yet assembled)."""
        ctx = ctypes.c_void_p()
        st = self.lib.ucg_deck_create(self.h, device, ctypes.byref(ctx))
        if st:
            raise UcgError(st, f"ucg_deck_create: {self.lib.ucg_strerror(st).decode()}")
        i = self.info
        return Simulation.adopt(ctx, i["mu"], i["lambda"], self.driver, i["n_rect"], i["n_tri"], i["n_vol"])

    def init_state(self, sim):
        y = np.zeros(sim.state_len)
        sim._check(self.lib.ucg_deck_init_state(self.h, sim.ctx, y.ctypes.data_as(_dp)), "init_state")
        return y

    def run(self, wdir=None, epsilon=1.0e-6, maximum_step=None, maximum_iterations=1000000,
            okada_mode=_lib.UCG_OKADA_REF32IO, precision=_lib.UCG_PREC_FP64, device=0, chunk=4096, verbose=False,
            hm_eta=0.0, hm_eps=0.0, hm_leaf=0):
        """The reference's main program on the device; writes time.txt, the
        observation-state and observation-point files into wdir (default: the
        deck's output directory).  precision UCG_PREC_HMATRIX builds the
        hierarchical K (hm_eta, hm_eps, hm_leaf; 0 for the defaults) instead
        of the dense one.  Returns (iterations, final time)."""
        o = _lib.RunOptions(epsilon, 1.7976931348623157e308 if maximum_step is None else maximum_step,
                            maximum_iterations, okada_mode, precision, device, chunk,
                            None if wdir is None else os.fspath(wdir).encode(), int(verbose), float(hm_eta),
                            float(hm_eps), int(hm_leaf))
        it, t = ctypes.c_long(), ctypes.c_double()
        st = self.lib.ucg_deck_run(self.h, ctypes.byref(o), ctypes.byref(it), ctypes.byref(t))
        if st:
            raise UcgError(st, f"ucg_deck_run: {self.lib.ucg_strerror(st).decode()}")
        return it.value, t.value


def _g(v):
    return repr(float(v))


def write_deck(cfg, wdir="output", driver=None, obs_patches=(), obs_volumes=(), obs_points=(), events=()):
    """Deck text for a configuration of unicycle_b200.configs (mesh, friction,
    and for coupled configs volumes and rheology), in the section order of the
    reference's init(); values with 17 significant digits.  obs_points:
    sequence of (name, (x1, x2, x3)); events: perturbation times after the
    first (which is at t = 0)."""
    m, fr = cfg["mesh"], cfg["friction"]
    driver = driver or ("viscouscycles" if "vol" in m else "ratestate")
    out = [f"# output directory", wdir, "# elastic moduli (lambda, mu)", f"{_g(cfg['lam'])} {_g(cfg['mu'])}",
           "# time interval", _g(cfg.get("t_end", 1.0))]
    k = 0
    rect = m.get("rect")
    nr = 0 if rect is None else len(rect[1])
    out += ["# number of rectangular patches", str(nr)]
    if nr:
        x, L, W, st, dp = rect
        out.append("#  n  Vpl  x1  x2  x3  length  width  strike  dip  rake")
        for i in range(nr):
            out.append(" ".join([str(i + 1), _g(fr["Vpl"][i])] + [_g(c) for c in x[i]] +
                                [_g(L[i]), _g(W[i]), _g(np.degrees(st[i])), _g(np.degrees(dp[i])),
                                 _g(np.degrees(fr["rake"][i]))]))
        out += ["# number of frictional rectangular patches", str(nr)]
        for i in range(nr):
            out.append(" ".join([str(i + 1)] + [_g(fr[q][i]) for q in ("mu0", "sig", "a", "b", "L", "Vo",
                                                                        "damping")]))
        k = nr
    tri = m.get("tri")
    nt = 0 if tri is None else len(tri[0])
    out += ["# number of triangular patches", str(nt)]
    if nt:
        i1, i2, i3, v = tri
        for i in range(nt):
            out.append(f"{i + 1} {_g(fr['Vpl'][k + i])} {int(i1[i])} {int(i2[i])} {int(i3[i])} "
                       f"{_g(np.degrees(fr['rake'][k + i]))}")
        out += ["# number of vertices", str(len(v))]
        for j in range(len(v)):
            out.append(" ".join([str(j + 1)] + [_g(c) for c in v[j]]))
        out += ["# number of frictional triangular patches", str(nt)]
        for i in range(nt):
            out.append(" ".join([str(i + 1)] + [_g(fr[q][k + i]) for q in ("mu0", "sig", "a", "b", "L", "Vo",
                                                                            "damping")]))
    if driver == "viscouscycles":
        vol = m.get("vol")
        nv = 0 if vol is None else len(vol[1])
        out += ["# number of cuboid strain volumes", str(nv)]
        if nv:
            x, L, T, W, st = vol
            rh = cfg["rheology"]
            ebg = np.asarray(rh["ebg"]).reshape(nv, 6)
            for i in range(nv):
                out.append(" ".join([str(i + 1)] + [_g(e) for e in ebg[i]] + [_g(c) for c in x[i]] +
                                    [_g(L[i]), _g(W[i]), _g(T[i]), _g(np.degrees(st[i])), "90"]))
            out += ["# number of nonlinear Maxwell strain volumes", str(nv)]
            for i in range(nv):
                out.append(" ".join([str(i + 1)] + [_g(rh[q][i]) for q in ("nGm", "gammadot0m", "npowerm", "nQm",
                                                                            "nRm")]))
            if "To" in rh:
                out += ["# number of thermal strain volumes", str(nv)]
                for i in range(nv):
                    out.append(f"{i + 1} {_g(rh.get('rhoc', np.ones(nv))[i])} {_g(rh['To'][i])}")
            else:
                out += ["# number of thermal strain volumes", "0"]
    out += ["# number of observation patches", str(len(obs_patches))]
    out += [f"{j + 1} {int(e)}" for j, e in enumerate(obs_patches)]
    if driver == "viscouscycles":
        out += ["# number of observation volumes", str(len(obs_volumes))]
        out += [f"{j + 1} {int(e)}" for j, e in enumerate(obs_volumes)]
    out += ["# number of observation points", str(len(obs_points))]
    out += [f"{j + 1} {name} {_g(x[0])} {_g(x[1])} {_g(x[2])}" for j, (name, x) in enumerate(obs_points)]
    out += ["# number of perturbations", str(len(events) + 1 if len(events) else 0)]
    out += [_g(t) for t in events]
    return "\n".join(out) + "\n"
