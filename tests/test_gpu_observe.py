"""GPU tests of the output path: the observation-point displacement kernels O
assembled on the device (buildO, greens.f90:302-462) against the oracle's
restatements of computeDisplacementOkada92 / Nikkhoo15 /
VerticalStrainVolume, and the device recorder (export / exportPoints,
ratestate.f90:405-537, viscouscycles.f90:521-633) against the host-driven
step loop.

Tolerances: Okada FP64 and Nikkhoo-Walter columns agree with the binary64
oracle to 1e-11 of the observation point's largest entry (the device contracts
products into FMAs, the oracle does not); REF32IO columns are REAL*4 outputs
and may differ by one binary32 rounding; volume columns are compared with the
oracle's 80-bit evaluation of the same integrals at 1e-9."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _point_scaled_err(O, ref):
    nobs = ref.shape[0] // 3
    sc = np.abs(ref).reshape(nobs, -1).max(axis=1)
    return np.max(np.abs(O - ref).reshape(nobs, -1).max(axis=1) / sc)


def _obs_points(rng, n, lo, hi, surface_frac=0.5):
    x = rng.uniform(lo, hi, size=(n, 3))
    x[: int(n * surface_frac), 2] = 0.0
    return x


@pytest.mark.parametrize("mode", [0, 1])
def test_build_o_rectangles(ucg, oracle_lib, mode):
    from unicycle_b200 import configs
    c = configs.cfg1(nx=16, nz=8)
    sim = ucg.Simulation(c["mu"], c["lam"])
    configs.build(sim, c)
    rng = np.random.default_rng(3)
    xo = _obs_points(rng, 40, [-10e3, 500.0, 0.0], [30e3, 15e3, 15e3])
    xo[::2, 1] *= -1.0                       # both sides of the fault, never on its plane
    sim.set_observation_points(xo)
    sim.buildO(mode)
    O = sim.copy_O()
    ref = oracle_lib.Mesh(c["mu"], c["lam"], rect=c["mesh"]["rect"], okada_mode=mode).build_o(xo)
    assert O.shape == ref.shape == (120, 2 * 128)
    assert np.all(np.isfinite(O))
    err = _point_scaled_err(O, ref)
    print(f"mode {mode}: max point-scaled error {err:.2e}; build {sim.observation_info()['build_ms']:.3f} ms")
    assert err < (2.5e-7 if mode == 1 else 1e-11)
    if mode == 1:   # REAL*4 outputs: the down component is a binary32 value
        assert np.array_equal(O[2::3], O[2::3].astype(np.float32).astype(np.float64))
    sim.close()


def test_build_o_triangles(ucg, oracle_lib):
    from unicycle_b200 import configs
    c = configs.cfg2(nx=8, nz=6)
    i1, i2, i3, v = c["mesh"]["tri"]
    sim = ucg.Simulation(c["mu"], c["lam"])
    sim.set_triangles(i1, i2, i3, v)
    sim.buildG()
    lo, hi = v.min(axis=0) - 5e3, v.max(axis=0) + 5e3
    rng = np.random.default_rng(4)
    xo = _obs_points(rng, 48, [lo[0], lo[1], 0.0], [hi[0], hi[1], hi[2]])
    sim.set_observation_points(xo)
    sim.buildO()
    O = sim.copy_O()
    ref = oracle_lib.Mesh(c["mu"], c["lam"], tri=(v, i1, i2, i3)).build_o(xo)
    assert np.all(np.isfinite(O))
    err = _point_scaled_err(O, ref)
    print(f"triangles: max point-scaled error {err:.2e}")
    assert err < 1e-11
    sim.close()


def test_build_o_volumes_and_split(ucg, oracle_lib):
    """Coupled fault + volumes: O against the oracle, and the total / faulting /
    flow displacement sets of a state against the host partition of O (the
    reference's buildO puts a volume's vertical column into Of)."""
    from unicycle_b200 import configs
    c = configs.cfg3(nxf=8, nzf=4, nxv=4, nyv=2, nzv=2)
    sim = ucg.Simulation(c["mu"], c["lam"], driver="viscouscycles")
    configs.build_coupled(sim, c)
    rng = np.random.default_rng(5)
    xo = _obs_points(rng, 24, [-20e3, 700.0, 0.0], [80e3, 40e3, 25e3])
    xo[1::2, 1] *= -1.0
    sim.set_observation_points(xo)
    sim.buildO()
    O = sim.copy_O()
    M = oracle_lib.Mesh(c["mu"], c["lam"], rect=c["mesh"]["rect"], vol=c["mesh"]["vol"])
    ref = M.build_o(xo)
    nf = 2 * c["n_patch"]
    assert np.all(np.isfinite(O))
    e_f = _point_scaled_err(O[:, :nf], ref[:, :nf])
    e_v = _point_scaled_err(O[:, nf:], ref[:, nf:])
    print(f"fault columns {e_f:.2e}, volume columns {e_v:.2e}")
    assert e_f < 1e-11 and e_v < 1e-9
    info = sim.observation_info()
    assert info["per_point"] == 9 and info["nobs"] == len(xo)

    K = sim.copy_G()
    y = configs.coseismic_preload(K, c)
    y[7 * c["n_patch"]:] += rng.standard_normal(len(y) - 7 * c["n_patch"]) * 1e-6
    d, df, dl = sim.displacements(y)
    u = np.concatenate([y[: 7 * c["n_patch"]].reshape(-1, 7)[:, :2].ravel(),
                        y[7 * c["n_patch"]:].reshape(-1, 12)[:, :6].ravel()])
    Of, Ol = O.copy(), O.copy()
    Of[:, nf:] = 0.0
    Of[2::3, nf:] = O[2::3, nf:]
    Ol[:, :nf] = 0.0
    Ol[2::3, :] = 0.0
    for got, want in ((d, O @ u), (df, Of @ u), (dl, Ol @ u)):
        want = want.reshape(-1, 3)
        assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want)) + 1e-300
    assert np.all(dl[:, 2] == 0.0)
    sim.close()


def test_recorder_matches_step_loop(ucg, oracle_lib):
    """Records written on the device at the start of every accepted step hold
    the time, the previous dt_done, the listed elements' state and rate, and O u
    -- the same values the host-driven ucg_step loop sees; ucg_run on a second
    context records the same trajectory."""
    from unicycle_b200 import configs
    c = configs.cfg1(nx=16, nz=8)
    xo = np.array([[5e3, 2e3, 0.0], [12e3, -3e3, 0.0], [20e3, 6e3, 1e3]])
    elems = [0, 37, 100]

    def make():
        sim = ucg.Simulation(c["mu"], c["lam"])
        configs.build(sim, c)
        sim.set_observation_points(xo)
        sim.buildO()
        return sim

    sim = make()
    O = sim.copy_O()
    sim.record(every=1, elements=elems, capacity=1000)
    t, y, dt = 0.0, c["y0"].copy(), c["dt0"]
    seen = []
    for _ in range(40):
        t1, y1, dydt, dt, dt_done, _ = sim.step(t, y, dt)
        seen.append((t, y.copy(), dydt.copy(), dt_done))
        t, y = t1, y1
    R = sim.records()
    assert len(R["time"]) == 40 and R["lost"] == 0
    for i, (ti, yi, dyi, _) in enumerate(seen):
        assert R["time"][i] == ti
        if i > 0:
            assert R["dt_done"][i] == seen[i - 1][3]
        for j, e in enumerate(elems):
            assert np.array_equal(R["state"][i, j, :7], yi[7 * e: 7 * e + 7])
            assert np.array_equal(R["rate"][i, j, :7], dyi[7 * e: 7 * e + 7])
        u = yi.reshape(-1, 7)[:, :2].ravel()
        want = (O @ u).reshape(-1, 3)
        assert np.max(np.abs(R["displacement"][i] - want)) <= 1e-12 * np.max(np.abs(want))
        assert np.array_equal(R["displacement"][i], sim.displacements(yi)[0])
    sim.close()

    # the same trajectory through ucg_run (device loop), every 4th step, small ring
    sim2 = make()
    sim2.set_state(c["y0"], 0.0, c["dt0"])
    sim2.record(every=4, elements=elems, capacity=3)
    sim2.run(1e30, 40)
    R2 = sim2.records()
    # 10 records were written (steps 0, 4, ..., 36); the ring kept the last 3
    assert R2["lost"] == 7 and len(R2["time"]) == 3
    for k, i in enumerate((28, 32, 36)):
        assert R2["time"][k] == seen[i][0]
        assert np.array_equal(R2["state"][k, :, :7], np.stack([seen[i][1][7 * e: 7 * e + 7] for e in elems]))
        assert np.array_equal(R2["displacement"][k], R["displacement"][i])
    sim2.close()
