"""Batched ensembles: the tensor-core contraction T = K V against FP64 on the same
inputs, its determinism and column independence, and ensemble Runge-Kutta
attempts against the single-instance FP64 integrator (which the oracle pins).

Error bound of the contraction: K and V are each held as fp16 hi + 2^-11 lo
pairs with a power-of-two scale per 128 x 64 block of K and per 64-source
block of each instance's V, so every product carries a relative error of about
2^-21 (both residuals; the dropped lo*lo term is 2^-44) for entries above
2^-14 of their block's largest, and every k-block's FP32 partial sum is added
into register sums with round-to-nearest; the test asks
|T - K V| <= 1e-5 (|K| |V|) entry by entry.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BOUND = 1.0e-5


def _small_cfg(shapes=((16, 8), (24, 8)), n_sets=40, seed=11):
    from unicycle_b200 import configs
    return configs.cfg4(shapes=shapes, n_sets=n_sets, size=1250.0, seed=seed)


def _geometry_sims(ucg, cfg):
    from unicycle_b200 import configs
    sims = []
    for g in cfg["geoms"]:
        sim = ucg.Simulation(g["mu"], g["lam"])
        configs.build(sim, g)
        sims.append(sim)
    return sims


def _ensemble(ucg, cfg, sims, sets=None):
    ens = ucg.Ensemble()
    for gi, (g, sim) in enumerate(zip(cfg["geoms"], sims)):
        ens.add_geometry(sim, len(g["sets"]))
        order = range(len(g["sets"])) if sets is None else sets[gi]
        for i, j in enumerate(order):
            fr = g["sets"][j]
            ens.set_friction(gi, i, fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"],
                             fr["Vo"], fr["damping"])
            ens.set_state(gi, i, g["y0s"][j], 0.0, cfg["dt0"])
    ens.set_tolerance(cfg["epsilon"])
    return ens


def _check_contraction(K, V, T, bound=BOUND):
    ref = V @ K.T
    mag = np.abs(V) @ np.abs(K).T
    ratio = np.abs(T - ref) / np.maximum(mag, 1e-300)
    assert np.all(np.isfinite(T))
    assert ratio.max() < bound, ratio.max()
    return ratio.max()


def test_contraction_matches_fp64(ucg):
    cfg = _small_cfg()
    sims = _geometry_sims(ucg, cfg)
    ens = _ensemble(ucg, cfg, sims)
    rng = np.random.default_rng(5)
    worst = []
    for gi, sim in enumerate(sims):
        K = sim.copy_G()
        ninst = len(cfg["geoms"][gi]["sets"])
        # slip-rate deficits over many decades, both signs
        V = rng.standard_normal((ninst, K.shape[1])) * 10.0 ** rng.uniform(-12, 0, (ninst, 1))
        T = ens.matvec(gi, V)
        worst.append(_check_contraction(K, V, T))
    print("max |T - KV| / (|K||V|):", worst)
    # the increments' form reads K hi only: error up to the fp16 unit roundoff 2^-11
    K = sims[0].copy_G()
    V = rng.standard_normal((len(cfg["geoms"][0]["sets"]), K.shape[1]))
    r2 = _check_contraction(K, V, ens.matvec(0, V, terms=2), bound=1e-3)
    print("two-term form: max |T - KV| / (|K||V|):", r2)
    for s in sims:
        s.close()
    ens.close()


def test_contraction_plans_deterministic_and_column_independent(ucg):
    from unicycle_b200 import _lib
    cfg = _small_cfg(shapes=((24, 8), (16, 12)), n_sets=70)
    sims = _geometry_sims(ucg, cfg)
    ens = _ensemble(ucg, cfg, sims)
    K = sims[1].copy_G()
    rng = np.random.default_rng(6)
    V = rng.standard_normal((70, K.shape[1]))
    plans = [(64, _lib.UCG_ENS_STREAM_K, 0), (64, _lib.UCG_ENS_SPLIT_LPT, 4), (32, _lib.UCG_ENS_SPLIT_LPT, 0),
             (32, _lib.UCG_ENS_STREAM_K, 0)]
    # 128-instance tiles are for hierarchical geometries only
    with pytest.raises(ucg.UcgError):
        ens.plan(128, _lib.UCG_ENS_STREAM_K, 0)
    results = []
    for ni, kind, chunk in plans:
        ens.plan(ni, kind, chunk)
        T1 = ens.matvec(1, V)
        T2 = ens.matvec(1, V)
        assert np.array_equal(T1, T2), (ni, kind, chunk)
        _check_contraction(K, V, T1)
        # instance 3's column does not depend on the other instances
        W = V.copy()
        W[np.arange(70) != 3] = rng.standard_normal((69, K.shape[1]))
        T3 = ens.matvec(1, W)
        assert np.array_equal(T3[3], T1[3]), (ni, kind, chunk)
        results.append(T1)
    report = ens.tune(reps=2)
    assert "chosen:" in report
    _check_contraction(K, V, ens.matvec(1, V))
    for s in sims:
        s.close()
    ens.close()


def test_ensemble_attempt_matches_fp64_integrator(ucg):
    """One attempt of every instance against one main-loop step of the FP64
    single-instance integrator from the same state: identical accepted step and
    time, the next step size within 5 % (the error estimate carries the
    increments' rounding), traction increments within the
    contraction's bound h 1e-4 (|K| |v|) and the other increments within 1e-3 of
    their FP64 scale."""
    cfg = _small_cfg()
    sims = _geometry_sims(ucg, cfg)
    ens = _ensemble(ucg, cfg, sims)
    assert ens.run(1.0e30, 1) == 1
    for gi, (g, sim) in enumerate(zip(cfg["geoms"], sims)):
        n = g["n_patch"]
        for i in (0, 7, len(g["sets"]) - 1):
            fr = g["sets"][i]
            sim.set_friction(fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"],
                             fr["damping"])
            y0 = g["y0s"][i]
            t64, y64, _, dn64, dd64, nrej = sim.step(0.0, y0, cfg["dt0"])
            y, t, dn, acc, rej, st = ens.get_state(gi, i)
            assert st == 0 and acc == 1 and rej == 0 and nrej == 0
            assert t == t64 == cfg["dt0"]
            assert abs(dn - dn64) <= 0.05 * dn64, (dn, dn64)
            d64 = (y64 - y0).reshape(n, 7)
            d = (y - y0).reshape(n, 7)
            Y = y0.reshape(n, 7)
            V, rake = 10.0 ** Y[:, 6], np.arctan2(Y[:, 3], Y[:, 2])
            v = np.empty(2 * n)
            v[0::2] = V * np.cos(rake) - fr["Vpl"] * np.cos(fr["rake"])
            v[1::2] = V * np.sin(rake) - fr["Vpl"] * np.sin(fr["rake"])
            # the contraction's bound over one step, plus the rounding of y + increment
            bound = cfg["dt0"] * BOUND * (np.abs(sim.copy_G()) @ np.abs(v)).reshape(n, 3)
            bound += 2.0 * np.spacing(np.abs(Y[:, 2:5]))
            assert np.all(np.abs(d[:, 2:5] - d64[:, 2:5]) <= bound), (gi, i)
            scale = np.maximum(np.abs(d64).max(axis=0), 1e-300)
            err = (np.abs(d - d64) / scale).max(axis=0)
            assert err[[0, 1, 5, 6]].max() < 1e-3, (gi, i, err)
    for s in sims:
        s.close()
    ens.close()


def _fp64_first_event(sim, y0, dt0, eps, von=1.0e-3, max_steps=20000):
    """Start time of the first main-loop step whose starting max slip rate is
    >= von, stepping the FP64 single-instance integrator; also the step count."""
    t, y, dn = 0.0, y0.copy(), dt0
    n = len(y0) // 7
    for k in range(max_steps):
        if 10.0 ** y.reshape(n, 7)[:, 6].max() >= von:
            return t, k
        t, y, _, dn, _, _ = sim.step(t, y, dn)
    return None, max_steps


def test_ensemble_event_onset_matches_fp64_integrator(ucg):
    """Run instances of a small fault through their first earthquake in the
    ensemble (tensor-core contraction, anchored stages) and with the FP64
    single-instance integrator: the onset times agree within 1e-4 relative
    (the reference-level criterion is 0.1 %), and the ensemble needs about the
    same number of steps."""
    cfg = _small_cfg(shapes=((16, 8),), n_sets=16)
    sims = _geometry_sims(ucg, cfg)
    ens = _ensemble(ucg, cfg, sims)
    sim = sims[0]
    g = cfg["geoms"][0]
    ens.set_event_threshold(1.0e-3, 1.0e-4)
    t_end = 0.0
    for i in (0, 5, 15):
        fr = g["sets"][i]
        sim.set_friction(fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"],
                         fr["damping"])
        sim.set_tolerance(cfg["epsilon"])
        t64, steps64 = _fp64_first_event(sim, g["y0s"][i], cfg["dt0"], cfg["epsilon"])
        assert t64 is not None, i
        t_end = max(t_end, 1.05 * t64)
        g.setdefault("fp64_onsets", {})[i] = (t64, steps64)
    ens.run(t_end, 60000)
    for i, (t64, steps64) in g["fp64_onsets"].items():
        ne, tf = ens.events(0, i)
        y, t, dn, acc, rej, st = ens.get_state(0, i)
        print(f"instance {i}: onset fp64 {t64:.9e} ({steps64} steps)  ensemble {tf:.9e}  "
              f"rel {abs(tf - t64) / t64:.2e}; ensemble steps {acc}, rejected {rej}")
        assert st == 0 and ne >= 1
        assert abs(tf - t64) <= 1e-4 * t64
    ens.close()
    sim.close()


def test_ensemble_instances_are_independent(ucg):
    """Reordering the parameter sets reorders the trajectories bit for bit, and an
    instance with a non-finite state stops alone with UCG_E_NONFINITE."""
    cfg = _small_cfg(shapes=((16, 8),), n_sets=24)
    sims = _geometry_sims(ucg, cfg)
    perm = np.random.default_rng(1).permutation(24)
    a = _ensemble(ucg, cfg, sims)
    b = _ensemble(ucg, cfg, sims, sets=[perm])
    bad = cfg["geoms"][0]["y0s"][perm[4]].copy()
    bad[6] = np.nan
    b.set_state(0, 4, bad, 0.0, cfg["dt0"])
    a.run(1.0e30, 150)
    b.run(1.0e30, 150)
    for i in range(24):
        ya, ta, _, acca, reja, sta = a.get_state(0, perm[i])
        yb, tb, _, accb, rejb, stb = b.get_state(0, i)
        if i == 4:
            assert stb == 5 and accb == 0
            continue
        assert sta == stb == 0
        assert (acca, reja, ta) == (accb, rejb, tb)
        assert np.array_equal(ya, yb)
    a.close()
    b.close()
    for s in sims:
        s.close()


def test_ensemble_run_stops_at_t_end(ucg):
    from unicycle_b200 import configs
    cfg = _small_cfg(shapes=((16, 8), (8, 8)), n_sets=8)
    sims = _geometry_sims(ucg, cfg)
    ens = _ensemble(ucg, cfg, sims)
    t_end = 0.05 * configs.YEAR
    ens.run(t_end, 100000)
    info = ens.info()
    assert info["active"] == 0 and info["launches"] > 0 and info["plan"] and info["accepted"] > 0
    for gi, g in enumerate(cfg["geoms"]):
        for i in range(len(g["sets"])):
            y, t, dn, acc, rej, st = ens.get_state(gi, i)
            assert st == 0 and t >= t_end and acc > 0
    # a later t_end continues from there
    ens.run(2 * t_end, 100000)
    for gi, g in enumerate(cfg["geoms"]):
        y, t, dn, acc, rej, st = ens.get_state(gi, 0)
        assert t >= 2 * t_end
    ens.close()
    for s in sims:
        s.close()


def test_host_launched_attempts_match_graph(ucg):
    """The attempt loop launched kernel by kernel from the host (for profilers)
    gives bit-identical trajectories to the single graph launch."""
    cfg = _small_cfg(shapes=((16, 8),), n_sets=8)
    sims = _geometry_sims(ucg, cfg)
    a = _ensemble(ucg, cfg, sims)
    b = _ensemble(ucg, cfg, sims)
    b.use_graph(False)
    a.run(1.0e30, 40)
    b.run(1.0e30, 40)
    ya, *ra = a.get_states(0)
    yb, *rb = b.get_states(0)
    assert np.array_equal(ya, yb)
    for x, y in zip(ra, rb):
        assert np.array_equal(x, y)
    a.close()
    b.close()
    for s in sims:
        s.close()


def test_contraction_long_k_range(ucg):
    """A fault of 8,448 rectangles (16,896 sources = 264 k-blocks of 64 per
    tile): every plan cuts its segments to at most 256 k-blocks, so one FP32
    accumulator never sums more than 16,384 products; both forms against FP64
    on the first 768 rows of K, determinism of each plan."""
    from unicycle_b200 import _lib, configs
    c = configs.cfg1(nx=128, nz=66)
    sim = ucg.Simulation(c["mu"], c["lam"])
    sim.set_rectangles(*c["mesh"]["rect"])
    sim.buildG()
    ninst = 64
    ens = ucg.Ensemble()
    ens.add_geometry(sim, ninst)
    Kr = sim.copy_G(0, 768)
    rng = np.random.default_rng(9)
    V = rng.standard_normal((ninst, Kr.shape[1])) * 1e-9
    mag = np.abs(V) @ np.abs(Kr).T
    for plan in [(64, _lib.UCG_ENS_STREAM_K, 0), (64, _lib.UCG_ENS_SPLIT_LPT, 0), (32, _lib.UCG_ENS_STREAM_K, 0)]:
        ens.plan(*plan)
        T = ens.matvec(0, V)
        assert np.array_equal(T, ens.matvec(0, V)), plan
        r3 = np.max(np.abs(T[:, :768] - V @ Kr.T) / mag)
        r2 = np.max(np.abs(ens.matvec(0, V, terms=2)[:, :768] - V @ Kr.T) / mag)
        print(plan, f"anchor {r3:.2e}, increment form {r2:.2e}")
        assert r3 < BOUND and r2 < 5e-3, plan
    ens.close()
    sim.close()
