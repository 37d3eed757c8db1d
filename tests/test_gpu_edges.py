"""Edge cases of the C ABI and of the kernels' tilings: refusals before anything
runs on the device (the reference STOPs in these places: a mesh with a bad
vertex index, a call out of order), the smallest model (one rectangle), and
sizes that fill no tile: fewer receiver rows than one 128-row M-tile, source
counts that end inside a 64-source k-block, fewer instances than one instance
tile, and split planes whose row stride is padded."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _err(ucg, fn, *a):
    with pytest.raises(ucg.UcgError) as ei:
        fn(*a)
    return ei.value


def test_refusals_before_launch(ucg):
    from unicycle_b200 import configs
    c = configs.cfg1(nx=3, nz=2)
    sim = ucg.Simulation(c["mu"], c["lam"])
    # nothing to assemble, nothing to integrate
    _err(ucg, sim.buildG)
    _err(ucg, sim.odefun, np.zeros(7))
    # a triangle that names a vertex past the list, and a degenerate one (1-based ids)
    v = np.array([[0.0, 0.0, 1.0e3], [1.0e3, 0.0, 1.0e3], [0.0, 1.0e3, 2.0e3]])
    _err(ucg, sim.set_triangles, [1], [2], [4], v)
    _err(ucg, sim.set_triangles, [1], [2], [2], v)
    # a rectangle of zero width
    x, L, W, strike, dip = c["mesh"]["rect"]
    W0 = W.copy()
    W0[2] = 0.0
    _err(ucg, sim.set_rectangles, x, L, W0, strike, dip)
    # the valid mesh still assembles in the same context
    configs.build(sim, c)
    assert sim.dims == (2 * c["n_patch"], 3 * c["n_patch"])
    sim.close()


def test_one_rectangle_odefun_matches_oracle(ucg, oracle_lib):
    from unicycle_b200 import configs
    c = configs.cfg1(nx=1, nz=1)
    sim = ucg.Simulation(c["mu"], c["lam"])
    configs.build(sim, c)
    G = sim.copy_G()
    assert G.shape == (3, 2)
    md = oracle_lib.Model(G, c["friction"])
    y = c["y0"].copy()
    dy, _ = sim.odefun(y)
    ref, _ = md.odefun(y)
    sc = np.maximum(np.abs(ref), 1e-300)
    assert np.max(np.abs(dy - ref) / sc) < 1e-10
    sim.close()


@pytest.mark.parametrize("nx,nz,ninst", [(7, 3, 3), (11, 5, 33), (23, 9, 5)])
def test_ragged_ensemble_contraction(ucg, nx, nz, ninst):
    """21 / 55 / 207 patches: 63 / 165 / 621 receiver rows (less than one, one
    and a half, almost five M-tiles) and 42 / 110 / 414 sources (k-blocks that
    end part-way), 3 / 33 / 5 instances (a partial instance tile, one past a
    32-wide tile)."""
    from unicycle_b200 import configs
    c = configs.cfg1(nx=nx, nz=nz)
    sim = ucg.Simulation(c["mu"], c["lam"])
    configs.build(sim, c)
    K = sim.copy_G()
    fr = c["friction"]
    ens = ucg.Ensemble()
    ens.add_geometry(sim, ninst)
    for i in range(ninst):
        ens.set_friction(0, i, fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"],
                         fr["damping"])
        ens.set_state(0, i, c["y0"], 0.0, c["dt0"])
    ens.set_tolerance(c["epsilon"])
    rng = np.random.default_rng(nx * 100 + ninst)
    V = rng.standard_normal((ninst, K.shape[1])) * 10.0 ** rng.uniform(-12, -6, (ninst, 1))
    T = ens.matvec(0, V)
    ref = V @ K.T
    mag = np.abs(V) @ np.abs(K).T
    assert T.shape == ref.shape
    assert np.all(np.isfinite(T))
    assert np.max(np.abs(T - ref) / np.maximum(mag, 1e-300)) < 1e-5
    # and the ensemble marches: attempts run, every instance alive
    ens.run(1e300, 20)
    y, t, _, acc, _, st = ens.get_states(0)
    assert np.all(st == 0) and np.all(acc > 0) and np.all(np.isfinite(y))
    ens.close()
    sim.close()


@pytest.mark.parametrize("form", ["split_pair", "split_bf16"])
def test_split_planes_with_padded_rows(ucg, form):
    """21 patches: 42 sources, so the split planes' rows are padded to 48
    columns; the split right-hand side agrees with the FP64 one."""
    from unicycle_b200 import configs
    c = configs.cfg1(nx=7, nz=3)
    sim = ucg.Simulation(c["mu"], c["lam"])
    configs.build(sim, c)
    y = c["y0"].copy()
    want, _ = sim.odefun(y)
    sim.set_precision(form)
    got, _ = sim.odefun(y)
    sim.set_precision(ucg.UCG_PREC_FP64)
    a, b = got.reshape(-1, 7), want.reshape(-1, 7)
    sc = np.maximum(np.abs(b).max(axis=0), 1e-300)
    # traction rates (columns 2-4) carry the planes' rounding; the rest is exact
    assert np.max(np.abs(a - b) / sc) < 1e-5
    sim.close()
