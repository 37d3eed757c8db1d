"""GPU tests of deck-driven runs: a context loaded from a deck assembles the
same K as the same configuration loaded through the Python API, and
ucg_deck_run (the reference's main program on the device) writes time.txt,
patch-/volume-*.dat and opts-*.dat whose lines hold, in the reference's
formats, the values the host-driven ucg_step loop sees."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rows(path, skip=0, w=19):
    """Fixed-width fields as Fortran writes them: the first 19 columns, then
    fields of w columns (a negative ES20.12E3 value fills its field, so
    columns, not blanks, separate the values)."""
    with open(path) as f:
        lines = f.read().splitlines()[skip:]
    rows = []
    for ln in lines:
        vals = [float(ln[:19])] + [float(ln[p:p + w]) for p in range(19, len(ln), w)]
        rows.append(vals)
    return lines, np.array(rows)


def test_deck_context_equals_api_context(ucg):
    from unicycle_b200 import Deck, configs, write_deck
    for c in (configs.cfg1(nx=8, nz=4), configs.cfg2(nx=6, nz=4)):
        d = Deck(write_deck(c))
        s1 = d.simulation()
        s1.buildG()
        s2 = ucg.Simulation(c["mu"], c["lam"])
        configs.build(s2, c)
        assert np.array_equal(s1.copy_G(), s2.copy_G())
        y1 = d.init_state(s1)
        assert np.array_equal(y1, s2.initStateVector())
        s1.close()
        s2.close()


def _step_loop(sim, y0, n, eps):
    sim.set_tolerance(eps)
    t, y, dt = 0.0, y0.copy(), 1.0e-3
    seen = []
    for _ in range(n):
        t1, y1, dydt, dt, dt_done, _ = sim.step(t, y, dt)
        seen.append((t, y.copy(), dydt.copy(), dt_done))
        t, y = t1, y1
    return seen


def test_deck_run_writes_reference_files(ucg, tmp_path):
    from unicycle_b200 import Deck, configs, write_deck
    c = configs.cfg1(nx=16, nz=8)
    pts = [("GPS1", (5000.0, 3000.0, 0.0)), ("ST2", (12000.0, -4000.0, 0.0))]
    d = Deck(write_deck(c, wdir=str(tmp_path), obs_patches=[1, 50], obs_points=pts))
    n = 60
    it, t_end = d.run(maximum_iterations=n, epsilon=1e-6, chunk=16, okada_mode=0)
    assert it == n

    sim = d.simulation()
    sim.buildG(0)
    sim.buildO(0)
    seen = _step_loop(sim, d.init_state(sim), n, 1e-6)

    lines, T = _rows(tmp_path / "time.txt", skip=1)
    assert lines[0] == " 0.000000000000E+00 1.000000000000E-03"
    assert all(len(ln) == 38 for ln in lines)
    assert T.shape == (n + 1, 2)
    want_t = np.array([s[0] for s in seen])
    want_dt = np.array([0.0] + [s[3] for s in seen[:-1]])
    np.testing.assert_allclose(T[1:, 0], want_t, rtol=1e-12)
    np.testing.assert_allclose(T[1:, 1], want_dt, rtol=1e-12)
    for e in (1, 50):
        lines, P = _rows(tmp_path / f"patch-{e:08d}.dat", w=20)
        assert P.shape == (n, 15) and all(len(ln) == 19 + 20 * 14 for ln in lines)
        ys = np.array([s[1][7 * (e - 1): 7 * e] for s in seen])
        rs = np.array([s[2][7 * (e - 1): 7 * e] for s in seen])
        np.testing.assert_allclose(P[:, 1:8], ys, rtol=1e-12, atol=1e-300)
        np.testing.assert_allclose(P[:, 8:], rs, rtol=1e-12, atol=1e-300)
    for k, (name, _) in enumerate(pts):
        lines, D = _rows(tmp_path / f"opts-{name}.dat")
        assert D.shape == (n, 4) and all(len(ln) == 19 * 4 for ln in lines)
        want = np.array([sim.displacements(s[1])[0][k] for s in seen])
        np.testing.assert_allclose(D[:, 1:], want, rtol=1e-12, atol=1e-15 * np.abs(want).max())
    sim.close()


def test_viscous_deck_run(ucg, tmp_path):
    from unicycle_b200 import Deck, configs, write_deck
    c = configs.cfg3(nxf=8, nzf=4, nxv=4, nyv=2, nzv=2)
    nf = c["n_patch"]
    pts = [("P1", (20000.0, 15000.0, 0.0))]
    d = Deck(write_deck(c, wdir=str(tmp_path), obs_patches=[3], obs_volumes=[2], obs_points=pts),
             driver="viscouscycles")
    n = 25
    it, _ = d.run(maximum_iterations=n, epsilon=1e-6, chunk=8, okada_mode=0)
    assert it == n
    sim = d.simulation()
    sim.buildG(0)
    sim.buildO(0)
    seen = _step_loop(sim, d.init_state(sim), n, 1e-6)
    lines, V = _rows(tmp_path / "volume-00000002.dat", w=20)
    assert V.shape == (n, 25) and all(len(ln) == 19 + 20 * 24 for ln in lines)
    o = 7 * nf + 12
    np.testing.assert_allclose(V[:, 1:13], np.array([s[1][o:o + 12] for s in seen]), rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(V[:, 13:], np.array([s[2][o:o + 12] for s in seen]), rtol=1e-12, atol=1e-300)
    lines, D = _rows(tmp_path / "opts-P1.dat")
    assert D.shape == (n, 10)
    for i, s in enumerate(seen):
        dd, df, dl = (a[0] for a in sim.displacements(s[1]))
        want = np.concatenate([dd, df, dl])
        np.testing.assert_allclose(D[i, 1:], want, rtol=1e-12, atol=1e-15 * np.abs(want).max())
    assert os.path.exists(tmp_path / "patch-00000003.dat")
    sim.close()


def test_deck_run_on_hierarchical_matrix(ucg, tmp_path):
    """A deck run on the hierarchical K (no dense K assembled) writes the files
    of the host-driven step loop on the same hierarchical K, line for line (the
    product is deterministic).  Against the dense run only the first steps are
    compared: the reference's step control follows the rounding residue of
    near-zero components at start-up, so any change of the product, even one
    ulp of K, moves the later step sequence."""
    from unicycle_b200 import Deck, configs, write_deck
    c = configs.cfg1(nx=32, nz=16)
    pts = [("GPS1", (5000.0, 3000.0, 0.0))]
    n = 40
    d = Deck(write_deck(c, wdir=str(tmp_path), obs_patches=[7], obs_points=pts))
    it, _ = d.run(maximum_iterations=n, epsilon=1e-6, chunk=16, okada_mode=0, precision=ucg.UCG_PREC_HMATRIX,
                  hm_leaf=16)
    assert it == n
    sim = d.simulation()
    sim.build_hmatrix(okada_mode=0, eta=2.0, eps=1e-6, leaf=16)
    sim.set_precision(ucg.UCG_PREC_HMATRIX)
    sim.set_observation_points([p for _, p in pts])
    sim.buildO(0)
    seen = _step_loop(sim, d.init_state(sim), n, 1e-6)
    _, T = _rows(tmp_path / "time.txt", skip=1)
    np.testing.assert_allclose(T[1:, 0], [s_[0] for s_ in seen], rtol=1e-12)
    _, P = _rows(tmp_path / "patch-00000007.dat", w=20)
    np.testing.assert_allclose(P[:, 1:8], np.array([s_[1][42:49] for s_ in seen]), rtol=1e-12, atol=1e-300)
    _, D = _rows(tmp_path / "opts-GPS1.dat")
    want = np.array([sim.displacements(s_[1])[0][0] for s_ in seen])
    np.testing.assert_allclose(D[:, 1:], want, rtol=1e-12, atol=1e-15 * np.abs(want).max())
    sim.close()
    # the dense run agrees over the first steps
    wd = tmp_path / "dense"
    wd.mkdir()
    Deck(write_deck(c, wdir=str(wd), obs_patches=[7], obs_points=pts)).run(
        maximum_iterations=n, epsilon=1e-6, chunk=16, okada_mode=0)
    _, Td = _rows(wd / "time.txt", skip=1)
    np.testing.assert_allclose(T[:4, 0], Td[:4, 0], rtol=1e-9)
