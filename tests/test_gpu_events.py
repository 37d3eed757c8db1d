"""GPU tests of coseismic perturbations (ucg_add_event / ucg_apply_perturbation):
the run lands exactly on a perturbation time, the state then jumps by the
slip / strain increment and by the stress change K u computed on the host from
the same K, the trajectory before the perturbation is untouched, and
re-setting the state re-arms pending perturbations.  The reference reads
perturbation times (in%event, viscouscycles.f90:2022-2049) without content;
the host-side K u is the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

YEAR = 3.15576e7


def _cfg1_sim(ucg):
    from unicycle_b200 import configs
    c = configs.cfg1(nx=16, nz=8)
    sim = ucg.Simulation(c["mu"], c["lam"])
    configs.build(sim, c)
    return c, sim


def _jump(K, np_, u, y):
    """y + the perturbation u (slip on components 0,1; K u on 2..4)"""
    y = y.copy()
    y[0:7 * np_:7] += u[0:2 * np_:2]
    y[1:7 * np_:7] += u[1:2 * np_:2]
    t = K @ u
    for c in range(3):
        y[2 + c:7 * np_:7] += t[c::3]
    return y


def test_apply_perturbation_now(ucg):
    c, sim = _cfg1_sim(ucg)
    K = sim.copy_G()
    np_ = c["n_patch"]
    rng = np.random.default_rng(2)
    slip = rng.uniform(0.0, 1.0, size=(np_, 2))
    sim.set_state(c["y0"], 0.0, c["dt0"])
    sim.apply_perturbation(slip=slip)
    y = sim.get_state()[0]
    want = _jump(K, np_, slip.ravel(), c["y0"])
    scale = np.abs(want).max()
    assert np.max(np.abs(y - want)) <= 1e-13 * scale
    sim.close()


def test_event_lands_and_jumps(ucg):
    c, sim = _cfg1_sim(ucg)
    _, ref = _cfg1_sim(ucg)
    K = sim.copy_G()
    np_ = c["n_patch"]
    t_e, t_end = 0.7 * YEAR, 1.5 * YEAR
    slip = np.zeros((np_, 2))
    slip[np_ // 4: np_ // 2, 0] = 0.01
    elems = list(range(0, np_, 8))
    cap = 50000
    for s, u in ((sim, slip), (ref, np.zeros_like(slip))):
        s.set_state(c["y0"], 0.0, c["dt0"])
        s.add_event(t_e, slip=u)
        s.record(every=1, elements=elems, capacity=cap)
        s.run(t_end, cap)
    R, Q = sim.records(), ref.records()
    k = int(np.searchsorted(R["time"], t_e))
    assert R["time"][k] == t_e and Q["time"][k] == t_e   # a step ends exactly on the perturbation
    # identical before the perturbation
    assert np.array_equal(R["state"][:k], Q["state"][:k]) and np.array_equal(R["time"][:k], Q["time"][:k])
    # the record at t_e shows the perturbed state: the zero-perturbation run's state plus the jump
    dy = _jump(K, np_, slip.ravel(), np.zeros(7 * np_)).reshape(np_, 7)[elems]
    want = Q["state"][k, :, :7] + dy
    assert np.max(np.abs(R["state"][k, :, :7] - want)) <= 1e-12 * np.abs(want).max()
    # the run continues past the perturbation to the end time
    assert R["lost"] == 0 and sim.get_state()[1] >= t_end
    print("steps before / after the perturbation:", k, len(R["time"]) - k)

    # setting the state again re-arms the perturbation; the rerun is identical
    sim.record(every=1, elements=elems, capacity=cap)
    sim.set_state(c["y0"], 0.0, c["dt0"])
    sim.run(t_end, cap)
    R2 = sim.records()
    assert np.array_equal(R2["time"], R["time"]) and np.array_equal(R2["state"], R["state"])
    sim.close()
    ref.close()


def test_event_at_start_is_the_coseismic_preload(ucg):
    """cfg3's initial state (uniform coseismic strike slip's stress change)
    is a perturbation at t = 0 of the unloaded state."""
    from unicycle_b200 import configs
    c = configs.cfg3(nxf=8, nzf=4, nxv=4, nyv=2, nzv=2)
    sim = ucg.Simulation(c["mu"], c["lam"], driver="viscouscycles")
    configs.build_coupled(sim, c)
    K = sim.copy_G()
    nf = c["n_patch"]
    pre = configs.coseismic_preload(K, c)
    slip = np.zeros((nf, 2))
    slip[:, 0] = c["coseismic_slip"]
    want = pre.copy()
    want[0:7 * nf:7] += c["coseismic_slip"]
    scale = np.abs(want).max()
    # applied now
    sim.set_state(c["y0"], 0.0, 1e-3)
    sim.apply_perturbation(slip=slip)
    assert np.max(np.abs(sim.get_state()[0] - want)) <= 1e-12 * scale
    # as a perturbation at t = 0: the first record of the run holds the perturbed state
    nv = c["n_vol"]
    sim.set_state(c["y0"], 0.0, 1e-3)
    sim.add_event(0.0, slip=slip)
    sim.record(every=1, elements=list(range(nf + nv)), capacity=4)
    sim.run(1.0e6, 1)
    R = sim.records()
    assert R["time"][0] == 0.0
    got = np.concatenate([R["state"][0, :nf, :7].ravel(), R["state"][0, nf:, :12].ravel()])
    assert np.max(np.abs(got - want)) <= 1e-12 * scale
    sim.close()
