"""The bounded device waits give up and report UCG_E_TIMEOUT without faulting
or hanging the GPU, and the context stays usable.

The failure is made by the tests' fault-injection hooks, not by a broken
kernel: the product's first CTA issues no copies, so the waits on its stages
wait for data that never comes (a flag that nothing sets) and give up after a
short limit (2 ms here instead of the normal 4 s); with nothing issued there is
no copy or MMA in flight when the CTA leaves.  Every other CTA finishes its
work normally.  The status comes back through the usual return codes.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UCG_E_TIMEOUT = 6
LIMIT_NS = 2_000_000


def test_traction_wait_timeout(ucg):
    from unicycle_b200 import configs
    c = configs.cfg1(nx=16, nz=8)
    sim = ucg.Simulation(c["mu"], c["lam"])
    configs.build(sim, c)
    want, _ = sim.odefun(c["y0"])
    sim.test_wait_timeout(LIMIT_NS, hold=True)
    with pytest.raises(ucg.UcgError) as ei:
        sim.odefun(c["y0"])
    assert ei.value.status == UCG_E_TIMEOUT
    with pytest.raises(ucg.UcgError) as ei:
        sim.step(0.0, c["y0"], c["dt0"])
    assert ei.value.status == UCG_E_TIMEOUT
    # back to normal: identical results, steps go on
    sim.test_wait_timeout(0, hold=False)
    got, _ = sim.odefun(c["y0"])
    assert np.array_equal(got, want)
    t, y, *_ = sim.step(0.0, c["y0"], c["dt0"])
    assert t > 0.0 and np.all(np.isfinite(y))
    sim.close()


def test_contraction_wait_timeout(ucg):
    from unicycle_b200 import configs
    c4 = configs.cfg4(shapes=((16, 8),), n_sets=8, size=1250.0, seed=4)
    g = c4["geoms"][0]
    sim = ucg.Simulation(g["mu"], g["lam"])
    configs.build(sim, g)
    ens = ucg.Ensemble()
    ens.add_geometry(sim, 8)
    V = np.random.default_rng(0).standard_normal((8, 2 * g["n_patch"]))
    want = ens.matvec(0, V)
    for i in range(8):
        fr = g["sets"][i]
        ens.set_friction(0, i, fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"],
                         fr["damping"])
        ens.set_state(0, i, g["y0s"][i], 0.0, c4["dt0"])
    ens.set_tolerance(c4["epsilon"])
    ens.test_wait_timeout(LIMIT_NS, hold=True)
    with pytest.raises(ucg.UcgError) as ei:
        ens.matvec(0, V)
    assert ei.value.status == UCG_E_TIMEOUT
    with pytest.raises(ucg.UcgError) as ei:
        ens.run(1e30, 3)
    assert ei.value.status == UCG_E_TIMEOUT
    # back to normal: the same contraction bit for bit, and attempts from fresh states
    ens.test_wait_timeout(0, hold=False)
    assert np.array_equal(ens.matvec(0, V), want)
    for i in range(8):
        ens.set_state(0, i, g["y0s"][i], 0.0, c4["dt0"])
    assert ens.run(1e30, 3) == 3
    _, t, _, acc, _, st = ens.get_states(0)
    assert np.all(st == 0) and np.all(acc >= 1)
    ens.close()
    sim.close()
