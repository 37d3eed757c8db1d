"""GPU tests of the hierarchical approximation of K (ucg_build_hmatrix):
the product H x against the dense FP64 K x of the same model, determinism,
the integrator driven through its first earthquake with H against FP64, and a
context that never holds the dense K.  The dense K assembled by the same pair
kernels (itself pinned to the oracle) is the reference here; the approximation
is held to a relative accuracy stated per test."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_hmatrix_product_rectangles(ucg):
    from unicycle_b200 import configs
    c = configs.cfg1(nx=64, nz=32)
    sim = ucg.Simulation(c["mu"], c["lam"])
    configs.build(sim, c)
    K = sim.copy_G()
    sim.build_hmatrix(eta=2.0, eps=1e-6, leaf=32)
    info = sim.hmatrix_info()
    print("rectangles 2048:", info)
    rng = np.random.default_rng(0)
    for _ in range(3):
        x = rng.standard_normal(K.shape[1])
        y = sim.hmatrix_matvec(x)
        err = _rel(y, K @ x)
        print(f"  |Hx - Kx| / |Kx| = {err:.2e}")
        assert err < 1e-6
    assert np.array_equal(sim.hmatrix_matvec(x), y)   # fixed summation order
    assert info["n_lowrank"] > 0 and info["compression"] > 2.0
    sim.close()


def test_hmatrix_product_triangles(ucg):
    from unicycle_b200 import configs
    c = configs.cfg2(nx=40, nz=20)
    i1, i2, i3, v = c["mesh"]["tri"]
    sim = ucg.Simulation(c["mu"], c["lam"])
    sim.set_triangles(i1, i2, i3, v)
    sim.buildG()
    K = sim.copy_G()
    sim.build_hmatrix(eta=2.0, eps=1e-6, leaf=32)
    info = sim.hmatrix_info()
    print("triangles 1600:", info)
    x = np.random.default_rng(1).standard_normal(K.shape[1])
    err = _rel(sim.hmatrix_matvec(x), K @ x)
    print(f"  |Hx - Kx| / |Kx| = {err:.2e}")
    assert err < 1e-6
    sim.close()


def _first_event(sim, y0, dt0, von=1.0e-3, max_steps=20000):
    t, y, dn = 0.0, y0.copy(), dt0
    n = len(y0) // 7
    for k in range(max_steps):
        if 10.0 ** y.reshape(n, 7)[:, 6].max() >= von:
            return t, k
        t, y, _, dn, _, _ = sim.step(t, y, dn)
    return None, max_steps


def test_hmatrix_event_onset_matches_fp64(ucg):
    from unicycle_b200 import configs
    cfg = configs.cfg4(shapes=((32, 16),), n_sets=2, size=1250.0, seed=11)
    g = cfg["geoms"][0]
    sim = ucg.Simulation(g["mu"], g["lam"])
    configs.build(sim, g)
    sim.build_hmatrix(eta=2.0, eps=1e-6, leaf=32)
    print(sim.hmatrix_info())
    fr = g["sets"][0]
    sim.set_friction(fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"], fr["damping"])
    sim.set_precision(ucg.UCG_PREC_FP64)
    t64, k64 = _first_event(sim, g["y0s"][0], cfg["dt0"])
    sim.set_precision(ucg.UCG_PREC_HMATRIX)
    th, kh = _first_event(sim, g["y0s"][0], cfg["dt0"])
    print(f"fp64 onset {t64:.9e} ({k64} steps); hmatrix {th:.9e} ({kh} steps); rel {abs(th - t64) / t64:.2e}")
    assert t64 is not None and th is not None
    assert abs(th - t64) <= 1e-4 * t64
    assert kh <= 1.2 * k64 + 20
    sim.close()


def test_hmatrix_without_dense_matrix(ucg):
    """A context that never assembles K: the right-hand side, steps and a
    perturbation run on the hierarchical matrix alone and agree with a dense
    context to the approximation's accuracy."""
    from unicycle_b200 import configs
    c = configs.cfg1(nx=32, nz=16)
    dense = ucg.Simulation(c["mu"], c["lam"])
    configs.build(dense, c)
    K = dense.copy_G()
    sim = ucg.Simulation(c["mu"], c["lam"])
    sim.set_rectangles(*c["mesh"]["rect"])
    fr = c["friction"]
    sim.set_friction(fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"], fr["damping"])
    sim.set_tolerance(c["epsilon"])
    sim.build_hmatrix(eta=2.0, eps=1e-6, leaf=16)
    sim.set_precision(ucg.UCG_PREC_HMATRIX)
    with pytest.raises(ucg.UcgError):
        sim.copy_G()
    y0 = c["y0"]
    d_h, _ = sim.odefun(y0)
    d_d, _ = dense.odefun(y0)
    np_ = c["n_patch"]
    for comp in range(7):
        a, b = d_h[comp::7], d_d[comp::7]
        assert np.max(np.abs(a - b)) <= 1e-6 * max(np.max(np.abs(b)), 1e-300), comp
    # a perturbation: the stress change comes from H u
    slip = np.zeros((np_, 2))
    slip[: np_ // 2, 0] = 0.05
    sim.set_state(y0, 0.0, c["dt0"])
    sim.apply_perturbation(slip=slip)
    y = sim.get_state()[0]
    t = K @ slip.ravel()
    want = y0.copy()
    want[0::7] += slip[:, 0]
    for q in range(3):
        want[2 + q::7] += t[q::3]
    assert np.max(np.abs(y - want)) <= 1e-7 * np.abs(want).max()
    # steps on the hierarchical matrix
    sim.set_state(y0, 0.0, c["dt0"])
    assert sim.run(1e30, 50) == 50
    sim.close()
    dense.close()


def test_hmatrix_split_matches_fp64(ucg):
    """The hierarchical K stored as bf16 hi + lo with anchored stages: the
    right-hand side within the split product's bound of the FP64 hierarchical
    one, and the first event's onset within 1e-4 of the FP64 integrator's."""
    from unicycle_b200 import configs
    cfg = configs.cfg4(shapes=((32, 16),), n_sets=2, size=1250.0, seed=11)
    g = cfg["geoms"][0]
    sim = ucg.Simulation(g["mu"], g["lam"])
    configs.build(sim, g)
    sim.build_hmatrix(eta=2.0, eps=1e-6, leaf=32)
    fr = g["sets"][0]
    sim.set_friction(fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"], fr["damping"])
    y0 = g["y0s"][0]
    sim.set_precision(ucg.UCG_PREC_HMATRIX)
    d64, _ = sim.odefun(y0)
    sim.set_precision(ucg.UCG_PREC_HMATRIX_SPLIT)
    dsp, _ = sim.odefun(y0)
    idx = np.concatenate([np.arange(q, len(y0), 7) for q in (2, 3, 4)])
    rel = np.max(np.abs(dsp[idx] - d64[idx])) / np.max(np.abs(d64[idx]))
    print(f"split vs FP64 hierarchical right-hand side: {rel:.2e}")
    assert rel < 1e-4
    sim.set_precision(ucg.UCG_PREC_FP64)
    t64, k64 = _first_event(sim, y0, cfg["dt0"])
    sim.set_precision(ucg.UCG_PREC_HMATRIX_SPLIT)
    ts, ks = _first_event(sim, y0, cfg["dt0"])
    print(f"fp64 onset {t64:.9e} ({k64} steps); hmatrix split {ts:.9e} ({ks} steps); rel {abs(ts - t64) / t64:.2e}")
    assert t64 is not None and ts is not None
    assert abs(ts - t64) <= 1e-4 * t64
    assert ks <= 1.5 * k64 + 20
    sim.close()
