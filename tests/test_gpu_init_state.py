"""ucg_init_state (initStateVector, fortran/3d/src/ratestate.f90:548-610 and
fortran/3d/src/viscouscycles.f90:710-820) against the oracle's orc_init_state
on the same parameters: both drivers, seeded per-patch friction with oblique
rakes, and volumes with a background strain rate and per-volume flow-law
constants.  The two evaluate the same closed forms in the same order, so they
agree to the last bit; the test allows 1 ulp."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _friction(rng, n):
    return dict(Vpl=10.0 ** rng.uniform(-9.5, -8.5, n), rake=rng.uniform(-np.pi, np.pi, n),
                mu0=rng.uniform(0.5, 0.7, n), sig=rng.uniform(10.0, 100.0, n), a=rng.uniform(0.005, 0.02, n),
                b=rng.uniform(0.002, 0.025, n), L=10.0 ** rng.uniform(-3, -1, n), Vo=np.full(n, 1e-6),
                damping=rng.uniform(1.0, 10.0, n))


def _close(got, want):
    tol = 4.5e-16 * np.maximum(np.abs(want), 1e-300)
    bad = np.abs(got - want) > tol
    assert not bad.any(), (np.flatnonzero(bad)[:8], got[bad][:4], want[bad][:4])


@pytest.mark.parametrize("driver", ["ratestate", "viscouscycles"])
def test_init_state_matches_oracle_faults(ucg, oracle_lib, driver):
    from unicycle_b200 import configs
    rng = np.random.default_rng(11)
    c = configs.cfg1(nx=6, nz=4)
    c2 = configs.cfg2(nx=3, nz=2)
    nr, nt = c["n_patch"], c2["n_patch"]
    fr = _friction(rng, nr + nt)
    sim = ucg.Simulation(c["mu"], c["lam"], driver=driver)
    sim.set_rectangles(*c["mesh"]["rect"])
    i1, i2, i3, v = c2["mesh"]["tri"]
    sim.set_triangles(i1, i2, i3, v)
    sim.set_friction(*(fr[k] for k in ("Vpl", "rake", "mu0", "sig", "a", "b", "L", "Vo", "damping")))
    got = sim.initStateVector()
    sim.close()
    want = oracle_lib.Model(None, fr, viscous=(driver == "viscouscycles")).init_state()
    assert got.shape == want.shape
    _close(got, want)


def test_init_state_matches_oracle_volumes(ucg, oracle_lib):
    from unicycle_b200 import configs
    rng = np.random.default_rng(12)
    c = configs.cfg3(nxf=4, nzf=2, nxv=2, nyv=2, nzv=2)
    nf, nv = c["n_patch"], c["n_vol"]
    fr = _friction(rng, nf)
    ebg = rng.normal(0.0, 1e-14, (nv, 6))
    ebg[0] = 0.0                                    # no background flow: zero initial stress
    vol = dict(ebg=ebg, gammadot0m=10.0 ** rng.uniform(-13, -11, nv), npowerm=rng.uniform(1.0, 3.5, nv),
               nGm=rng.uniform(1e4, 3e4, nv), nQm=rng.uniform(0.0, 2e5, nv), nRm=np.full(nv, 8.314),
               To=rng.uniform(800.0, 1600.0, nv))
    sim = ucg.Simulation(c["mu"], c["lam"], driver="viscouscycles")
    sim.set_rectangles(*c["mesh"]["rect"])
    sim.set_volumes(*c["mesh"]["vol"])
    sim.set_friction(*(fr[k] for k in ("Vpl", "rake", "mu0", "sig", "a", "b", "L", "Vo", "damping")))
    sim.set_rheology(vol["ebg"], vol["gammadot0m"], vol["npowerm"], nonlinear_maxwell=True)
    got = sim.initStateVector(vol["nGm"], vol["nQm"], vol["nRm"], vol["To"])
    sim.close()
    want = oracle_lib.Model(None, fr, vol=vol, viscous=True, nonlinear_maxwell=True).init_state()
    assert got.shape == want.shape == (7 * nf + 12 * nv,)
    assert np.all(want[7 * nf + 6:7 * nf + 12] == 0.0)
    _close(got, want)
