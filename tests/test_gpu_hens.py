"""Ensembles on the hierarchical K: the two-pass tensor-core contraction
T = H V (pass 1 Z = V_b X per rank stack, pass 2 [dense | U] [X ; Z] per row
leaf) against the FP64 hierarchical product of the same matrix, its
determinism and column independence, and the first event of ensemble
instances against the FP64 single-instance integrator.

Error bound of the contraction, entry by entry against |K| |V| (|K| the dense
matrix of the same model; the hierarchical matrix is within 1e-6 of it).  Two
planes: both passes split their operands into bf16 hi + lo (about 3 * 2^-16
relative per product) and Z is rounded to hi + lo once between them: 2e-4.
Three planes (the default): hi + mid + lo (24 bits; the products left out are
below 2^-24) with FP32 tensor-core sums over runs of at most 1,024 entries: 2e-6.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BOUND = 2.0e-4       # two planes
BOUND3 = 2.0e-6      # three planes


def _model(ucg, kind, leaf=32):
    from unicycle_b200 import configs
    if kind == "rect":
        c = configs.cfg1(nx=64, nz=32)
        sim = ucg.Simulation(c["mu"], c["lam"])
        configs.build(sim, c)
    else:
        c = configs.cfg2(nx=40, nz=20)
        i1, i2, i3, v = c["mesh"]["tri"]
        sim = ucg.Simulation(c["mu"], c["lam"])
        sim.set_triangles(i1, i2, i3, v)
        sim.buildG()
    K = sim.copy_G()
    sim.build_hmatrix(eta=2.0, eps=1e-6, leaf=leaf)
    sim.set_precision(ucg.UCG_PREC_HMATRIX)
    return sim, K


def _check(K, V, T, ref, bound):
    mag = np.abs(V) @ np.abs(K).T
    ratio = np.abs(T - ref) / np.maximum(mag, 1e-300)
    assert np.all(np.isfinite(T))
    assert ratio.max() < bound, ratio.max()
    return ratio.max()


@pytest.mark.parametrize("planes", [2, 3])
@pytest.mark.parametrize("kind", ["rect", "tri"])
def test_hier_contraction_matches_fp64_hmatrix(ucg, kind, planes):
    sim, K = _model(ucg, kind)
    ninst = 40
    ens = ucg.Ensemble()
    ens.set_hier_planes(planes)
    ens.add_geometry(sim, ninst)
    rng = np.random.default_rng(21)
    V = rng.standard_normal((ninst, K.shape[1])) * 10.0 ** rng.uniform(-12, 0, (ninst, 1))
    ref = np.stack([sim.hmatrix_matvec(v) for v in V])
    bound = BOUND if planes == 2 else BOUND3
    r3 = _check(K, V, ens.matvec(0, V), ref, bound)
    # slip rates of one sign: every run's sum grows with its length, and the
    # tensor core's truncation with it
    Va = np.abs(V)
    ra = _check(K, Va, ens.matvec(0, Va), np.stack([sim.hmatrix_matvec(v) for v in Va]), bound)
    # two planes: the increments' form reads the hi planes of H alone; three
    # planes: one form at every stage
    r2 = _check(K, V, ens.matvec(0, V, terms=2), ref, 1e-2 if planes == 2 else bound)
    print(kind, planes, ens.info()["plan"])
    print(f"{kind}, {planes} planes: max |T - HV| / (|K||V|) = {r3:.2e}, one-sign V {ra:.2e}; "
          f"two-term form {r2:.2e}")
    ens.close()
    sim.close()


def test_hier_planes_fixed_once_added(ucg):
    """The planes belong to the images: fixed by the first hierarchical
    geometry; three planes take no 128-instance tiles."""
    from unicycle_b200 import _lib
    sim, K = _model(ucg, "rect")
    ens = ucg.Ensemble()
    with pytest.raises(ucg.UcgError):
        ens.set_hier_planes(4)
    ens.add_geometry(sim, 8)
    ens.set_hier_planes(3)
    with pytest.raises(ucg.UcgError):
        ens.set_hier_planes(2)
    with pytest.raises(ucg.UcgError):
        ens.plan(128, _lib.UCG_ENS_STREAM_K, 0)
    ens.close()
    sim.close()


@pytest.mark.parametrize("planes", [2, 3])
def test_hier_contraction_deterministic_and_column_independent(ucg, planes):
    from unicycle_b200 import _lib
    sim, K = _model(ucg, "rect")
    ninst = 70
    ens = ucg.Ensemble()
    ens.set_hier_planes(planes)
    ens.add_geometry(sim, ninst)
    rng = np.random.default_rng(22)
    V = rng.standard_normal((ninst, K.shape[1]))
    ref = np.stack([sim.hmatrix_matvec(v) for v in V])
    for ni in ((32, 64, 128) if planes == 2 else (32, 64)):
        ens.plan(ni, _lib.UCG_ENS_STREAM_K, 0)
        T1 = ens.matvec(0, V)
        assert np.array_equal(T1, ens.matvec(0, V)), ni
        _check(K, V, T1, ref, BOUND if planes == 2 else BOUND3)
        W = V.copy()
        W[np.arange(ninst) != 5] = rng.standard_normal((ninst - 1, K.shape[1]))
        assert np.array_equal(ens.matvec(0, W)[5], T1[5]), ni
    ens.close()
    sim.close()


def test_hier_and_dense_geometries_in_one_ensemble(ucg):
    """A dense and a hierarchical geometry side by side: each contraction
    matches its own FP64 product."""
    from unicycle_b200 import configs
    sim_h, K = _model(ucg, "rect")
    c = configs.cfg1(nx=32, nz=16)
    sim_d = ucg.Simulation(c["mu"], c["lam"])
    configs.build(sim_d, c)
    Kd = sim_d.copy_G()
    ens = ucg.Ensemble()
    ens.add_geometry(sim_d, 24)
    ens.add_geometry(sim_h, 24)
    rng = np.random.default_rng(23)
    Vd = rng.standard_normal((24, Kd.shape[1]))
    Vh = rng.standard_normal((24, K.shape[1]))
    _check(Kd, Vd, ens.matvec(0, Vd), Vd @ Kd.T, 1e-4)
    _check(K, Vh, ens.matvec(1, Vh), np.stack([sim_h.hmatrix_matvec(v) for v in Vh]), BOUND3)
    ens.close()
    sim_h.close()
    sim_d.close()


def _fp64_first_event(sim, y0, dt0, von=1.0e-3, max_steps=20000):
    t, y, dn = 0.0, y0.copy(), dt0
    n = len(y0) // 7
    for k in range(max_steps):
        if 10.0 ** y.reshape(n, 7)[:, 6].max() >= von:
            return t, k
        t, y, _, dn, _, _ = sim.step(t, y, dn)
    return None, max_steps


def test_hier_ensemble_event_onset_matches_fp64(ucg):
    """Instances of a dipping fault through their first earthquake on the
    hierarchical K in the ensemble (anchored stages) against the dense FP64
    single-instance integrator: onsets within 1e-4 relative."""
    from unicycle_b200 import configs
    cfg = configs.cfg4(shapes=((32, 16),), n_sets=16, size=1250.0, seed=11)
    g = cfg["geoms"][0]
    dense = ucg.Simulation(g["mu"], g["lam"])
    configs.build(dense, g)
    hs = ucg.Simulation(g["mu"], g["lam"])
    configs.build(hs, g)
    hs.build_hmatrix(eta=2.0, eps=1e-6, leaf=32)
    hs.set_precision(ucg.UCG_PREC_HMATRIX)
    ens = ucg.Ensemble()
    ens.add_geometry(hs, len(g["sets"]))
    for i, fr in enumerate(g["sets"]):
        ens.set_friction(0, i, fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"],
                         fr["damping"])
        ens.set_state(0, i, g["y0s"][i], 0.0, cfg["dt0"])
    ens.set_tolerance(cfg["epsilon"])
    ens.set_event_threshold(1.0e-3, 1.0e-4)
    onsets = {}
    t_end = 0.0
    for i in (0, 9):
        fr = g["sets"][i]
        dense.set_friction(fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"],
                           fr["damping"])
        dense.set_tolerance(cfg["epsilon"])
        t64, k64 = _fp64_first_event(dense, g["y0s"][i], cfg["dt0"])
        assert t64 is not None
        onsets[i] = (t64, k64)
        t_end = max(t_end, 1.05 * t64)
    ens.run(t_end, 60000)
    print(ens.info()["plan"])
    for i, (t64, k64) in onsets.items():
        ne, tf = ens.events(0, i)
        y, t, dn, acc, rej, st = ens.get_state(0, i)
        print(f"instance {i}: onset fp64 {t64:.9e} ({k64} steps)  hierarchical ensemble {tf:.9e} "
              f"rel {abs(tf - t64) / t64:.2e}; steps {acc}, rejected {rej}")
        assert st == 0 and ne >= 1
        assert abs(tf - t64) <= 1e-4 * t64
    ens.close()
    hs.close()
    dense.close()


def test_hier_ensemble_rejects_wide_leaves(ucg):
    """Row leaves must fit one 128-row tile (at most 42 patches)."""
    from unicycle_b200 import configs
    c = configs.cfg1(nx=32, nz=16)
    sim = ucg.Simulation(c["mu"], c["lam"])
    sim.set_rectangles(*c["mesh"]["rect"])
    sim.build_hmatrix(eta=2.0, eps=1e-6, leaf=64)
    ens = ucg.Ensemble()
    with pytest.raises(ucg.UcgError):
        ens.add_geometry(sim, 8)
    ens.close()
    sim.close()
