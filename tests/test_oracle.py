"""CPU tests of the oracle: pins against the reference's own C (golden fixtures
and, where built, the live oracle/_ref library) and physical identities that
tie the Okada restatement to the reference Nikkhoo-Walter code."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
MU = LAM = 30.0e3


def rel_err(a, b, floor):
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))


def elem_scaled_err(G, ref, dof=3):
    """max |G - ref| / (max |ref| over the receiver element's rows).  Entries far
    below the element's traction scale are sums with heavy cancellation whose
    last bits are rounding noise in any FP64 evaluation (the reference's own C
    differs from an 80-bit evaluation there), so they are compared on the
    element's scale."""
    d = np.abs(G - ref)
    em = np.abs(ref).reshape(-1, dof, ref.shape[1]).max(axis=(1, 2))
    return np.max(d / np.repeat(em, dof)[:, None])


def test_nw15_restatement_matches_reference_pairs(oracle_lib):
    g = np.load(os.path.join(GOLD, "nw15_pairs.npz"))
    P, X, S = g["P"], g["X"], g["S"]
    worst = 0.0
    for k in range(len(X)):
        for j, (s, d) in enumerate(((1.0, 0.0), (0.0, 1.0))):
            a = oracle_lib.nw15_stress(X[k], P[k, 0], P[k, 1], P[k, 2], s, d, 0.0, MU, LAM)
            scale = np.max(np.abs(S[k, j]))
            worst = max(worst, np.max(np.abs(a - S[k, j])) / scale)
    # random points include near-singular geometry; the reference itself differs
    # from an 80-bit evaluation by up to ~4e-6 there
    assert worst < 1e-6, worst


def test_nw15_restatement_matches_reference_mesh(oracle_lib):
    g = np.load(os.path.join(GOLD, "nw15_mesh_G.npz"))
    M = oracle_lib.Mesh(MU, LAM, tri=(g["v"], g["i1"], g["i2"], g["i3"]))
    G = M.build_g()
    ref = g["G"]
    assert elem_scaled_err(G, ref) < 1e-12
    big = np.abs(ref) > 1e-2 * np.abs(ref).max()
    assert rel_err(G[big], ref[big], 0.0) < 1e-12


def test_nw15_live_reference(oracle_lib):
    if oracle_lib.ref_lib() is None:
        pytest.skip("reference C sources not present here")
    rng = np.random.default_rng(5)
    for _ in range(50):
        P = rng.uniform([-3e3, -3e3, 1e3], [3e3, 3e3, 6e3], size=(3, 3))
        x = rng.uniform([-8e3, -8e3, 0.5e3], [8e3, 8e3, 10e3])
        for s, d in ((1.0, 0.0), (0.0, 1.0)):
            a = oracle_lib.nw15_stress(x, *P, s, d, 0.0, MU, LAM)
            b = oracle_lib.nw15_stress_ref(x, *P, s, d, 0.0, MU, LAM)
            assert np.max(np.abs(a - b)) <= 1e-8 * np.max(np.abs(b))


def _rect_as_triangles(q, L, W, strike, dip):
    sv = np.array([np.cos(strike), np.sin(strike), 0.0])
    dv = np.array([np.sin(strike) * np.cos(dip), -np.cos(strike) * np.cos(dip), -np.sin(dip)])
    A = q
    B = q + L * sv
    C = q + L * sv - W * dv
    D = q - W * dv
    return (A, B, C), (A, C, D)


@pytest.mark.parametrize("dip_deg", [90.0, 60.0, 30.0])
def test_okada_equals_two_triangles(oracle_lib, dip_deg):
    """A rectangle is two triangles: the Okada restatement against the
    reference's own Nikkhoo-Walter code (or its restatement) away from edges.
    Strike 0: the reference's rotation of the gradient back from the strike
    frame (okada92.f90:172, uxzr = -cos*uxz + sin*uyz) has the opposite sign on
    the sin*uyz term from the chain rule, so for strike != 0 the reference's
    Okada stress differs from the two-triangle field; the restatement keeps the
    reference's expression (see test_okada_reference_uxz_rotation)."""
    nw = oracle_lib.nw15_stress_ref if oracle_lib.ref_lib() is not None else oracle_lib.nw15_stress
    q = np.array([0.0, 0.0, 2000.0])
    L, W, strike, dip = 3000.0, 2000.0, 0.0, np.radians(dip_deg)
    t1, t2 = _rect_as_triangles(q, L, W, strike, dip)
    rng = np.random.default_rng(7)
    worst = 0.0
    for _ in range(40):
        x = rng.uniform([-6e3, -6e3, 100.0], [9e3, 9e3, 9e3])
        for s, d in ((1.0, 0.0), (0.0, 1.0)):
            ok = oracle_lib.okada_stress(oracle_lib.OKADA_FP64, x, q, L, W, strike, dip, s, d, 0.0, MU, LAM)
            tr = nw(x, *t1, s, d, 0.0, MU, LAM) + nw(x, *t2, s, d, 0.0, MU, LAM)
            worst = max(worst, np.max(np.abs(ok - tr)) / np.max(np.abs(tr)))
    assert worst < 1e-9, worst


def test_okada_reference_uxz_rotation(oracle_lib):
    """For strike != 0 the restatement reproduces the reference's uxzr
    expression: the difference from the two-triangle field is exactly the stress
    of the doubled sin(strike)*uyz term in e13."""
    q = np.array([0.0, 0.0, 2000.0])
    L, W, strike, dip = 3000.0, 2000.0, np.radians(20.0), np.radians(60.0)
    t1, t2 = _rect_as_triangles(q, L, W, strike, dip)
    x = np.array([5000.0, -3000.0, 4000.0])
    ok = oracle_lib.okada_stress(0, x, q, L, W, strike, dip, 1.0, 0.0, 0.0, MU, LAM)
    tr = oracle_lib.nw15_stress(x, *t1, 1.0, 0.0, 0.0, MU, LAM) + oracle_lib.nw15_stress(x, *t2, 1.0, 0.0, 0.0, MU, LAM)
    # DC3D gradient entry uyz for this point (DC3D frame)
    cs, ss = np.cos(strike), np.sin(strike)
    X = (x[0] - q[0]) * cs + (x[1] - q[1]) * ss
    Y = (x[0] - q[0]) * ss - (x[1] - q[1]) * cs
    _, u = oracle_lib.dc3d(0, 2.0 / 3.0, X, Y, -x[2], q[2], np.degrees(dip), 0.0, L, -W, 0.0, 1.0, 0.0, 0.0)
    uyz = u[10]
    # reference: e13 = (uxzr + uzxr)/2 with uxzr carrying +sin*uyz instead of -sin*uyz
    d13 = 2.0 * MU * (ss * uyz)   # = 2 mu * (half of the 2 sin uyz difference)
    diff = ok - tr
    assert abs(diff[2] - d13) < 1e-9 * np.max(np.abs(tr))
    assert np.max(np.abs(diff[[0, 1, 3, 4, 5]])) < 1e-9 * np.max(np.abs(tr))


def test_okada_free_surface_traction_free(oracle_lib):
    q = np.array([0.0, 0.0, 1000.0])
    rng = np.random.default_rng(3)
    for _ in range(20):
        x = np.array([rng.uniform(-5e3, 5e3), rng.uniform(-5e3, 5e3), 0.0])
        for s, d in ((1.0, 0.0), (0.0, 1.0)):
            # strike 0: see test_okada_reference_uxz_rotation
            sig = oracle_lib.okada_stress(oracle_lib.OKADA_FP64, x, q, 2000.0, 1500.0, 0.0, 1.1, s, d, 0.0, MU, LAM)
            scale = np.max(np.abs(sig))
            assert np.max(np.abs(sig[[2, 4, 5]])) < 1e-9 * scale


def test_nw15_free_surface_traction_free(oracle_lib):
    P = [np.array([0.0, 0.0, 1000.0]), np.array([2000.0, 500.0, 1500.0]), np.array([500.0, 1500.0, 3000.0])]
    rng = np.random.default_rng(4)
    for _ in range(20):
        x = np.array([rng.uniform(-5e3, 5e3), rng.uniform(-5e3, 5e3), 0.0])
        for s, d in ((1.0, 0.0), (0.0, 1.0)):
            sig = oracle_lib.nw15_stress(x, *P, s, d, 0.0, MU, LAM)
            assert np.max(np.abs(sig[[2, 4, 5]])) < 1e-9 * np.max(np.abs(sig))


def test_okada_far_field_decay(oracle_lib):
    q = np.array([0.0, 0.0, 5000.0])
    sig1 = oracle_lib.okada_stress(0, np.array([0.0, 50e3, 5000.0]), q, 100.0, 100.0, 0.0, np.pi / 2, 1, 0, 0, MU, LAM)
    sig2 = oracle_lib.okada_stress(0, np.array([0.0, 100e3, 5000.0]), q, 100.0, 100.0, 0.0, np.pi / 2, 1, 0, 0, MU, LAM)
    ratio = np.max(np.abs(sig1)) / np.max(np.abs(sig2))
    assert 6.0 < ratio < 10.0   # ~ r^-3 (half-space corrections perturb it)


def test_okada_ref32io_close_to_fp64(oracle_lib):
    rng = np.random.default_rng(8)
    q = np.array([1000.0, -500.0, 1500.0])
    for _ in range(30):
        x = rng.uniform([-5e3, -5e3, 200.0], [5e3, 5e3, 6e3])
        a = oracle_lib.okada_stress(0, x, q, 1250.0, 1250.0, 0.4, 1.2, 1, 0, 0, MU, LAM)
        b = oracle_lib.okada_stress(1, x, q, 1250.0, 1250.0, 0.4, 1.2, 1, 0, 0, MU, LAM)
        assert np.max(np.abs(a - b)) <= 1e-5 * np.max(np.abs(a))


def test_okada_singular_edge_is_zero(oracle_lib):
    # DC3D rejects points on the fault edge (dc3d.f:69-73) and returns zeros
    ret, u = oracle_lib.dc3d(0, 2.0 / 3.0, 0.0, 0.0, -1.0, 1.0, 90.0, 0.0, 1.0, -1.0, 0.0, 1.0, 0.0, 0.0)
    assert ret == 1 and np.all(u == 0.0)


def test_rkck_fifth_order_local_error(oracle_lib):
    """Cash-Karp local error of the 5th-order solution scales as h^5 (the
    embedded 4th-order difference, yerr, as h^5 too)."""
    from unicycle_b200 import configs
    c = configs.cfg1(nx=4, nz=2)
    M = oracle_lib.Mesh(c["mu"], c["lam"], rect=c["mesh"]["rect"])
    G = M.build_g()
    md = oracle_lib.Model(G, c["friction"])
    y0 = c["y0"]
    dydt, _ = md.odefun(y0)
    errs = []
    for h in (2e6, 1e6):
        y1, yerr = md.rkck(y0, dydt, h)
        # reference solution with 64 substeps
        y = y0.copy()
        for _ in range(64):
            k, _ = md.odefun(y)
            y, _ = md.rkck(y, k, h / 64)
        errs.append(np.max(np.abs(y1 - y)))
    assert errs[0] / errs[1] > 20.0   # 2^5 = 32, loosely


def test_rkqs_controller_rejects_and_shrinks(oracle_lib):
    from unicycle_b200 import configs
    c = configs.cfg1(nx=8, nz=4)
    M = oracle_lib.Mesh(c["mu"], c["lam"], rect=c["mesh"]["rect"])
    md = oracle_lib.Model(M.build_g(), c["friction"])
    y0 = c["y0"]
    dydt, _ = md.odefun(y0)
    yscal = np.abs(y0) + np.abs(1e7 * dydt) + 1e-30
    rc, y1, hdid, hnext, nrej = md.rkqs(y0, dydt, yscal, 1e7, 1e-8)
    assert rc == 0 and nrej >= 1 and hdid < 1e7 and hnext > 0.0


def test_state_init_matches_reference_formula(oracle_lib):
    from unicycle_b200 import configs
    c = configs.cfg1(nx=4, nz=2)
    md = oracle_lib.Model(np.zeros((24, 16)), c["friction"])
    y = md.init_state()
    fr = c["friction"]
    tau = fr["sig"] * (fr["mu0"] + (fr["a"] - fr["b"]) * np.log(fr["Vpl"] / fr["Vo"])) - fr["damping"] * fr["Vpl"]
    assert np.allclose(y[2::7], tau * np.cos(fr["rake"]), rtol=1e-15)
    assert np.allclose(y[6::7], np.log10(0.99 * fr["Vpl"]), rtol=1e-15)


def test_reference_step_control_is_rounding_sensitive(oracle_lib):
    """Documents a property of the reference algorithm: on the symmetric
    strike-slip fault the RKQS error norm is set by state components that are
    zero analytically (dip slip, dip traction) and hold only rounding residue,
    so perturbing G by one ulp already moves the accepted step sizes by more
    than 1e-4 within a few steps.  History comparisons are therefore made
    against this envelope (tests/test_gpu_parity.py)."""
    from unicycle_b200 import configs
    c = configs.cfg1()
    G = oracle_lib.Mesh(c["mu"], c["lam"], rect=c["mesh"]["rect"]).build_g()

    def times(Gm):
        md = oracle_lib.Model(Gm, c["friction"])
        y, t, dt, out = c["y0"].copy(), 0.0, c["dt0"], []
        for _ in range(8):
            rc, t, y, _, dt, _, _ = md.step(t, y, dt, c["epsilon"])
            out.append(t)
        return np.array(out)

    rng = np.random.default_rng(0)
    Gp = G * (1.0 + rng.choice([-1.0, 0.0, 1.0], size=G.shape) * 2.220446049250313e-16)
    a, b = times(G), times(Gp)
    assert np.max(np.abs(a - b) / a) > 1e-4


# ---- strain volumes (Barbot, Moore & Lambert 2017) ---------------------------

NU = 0.25


def _sv(oracle_lib, x, q, L, T, W, th, eps):
    return oracle_lib.bml17_stress(np.asarray(x, float), np.asarray(q, float), L, T, W, th, eps, MU, NU)


@pytest.mark.parametrize("q", range(6))
def test_bml17_free_surface_traction_free(oracle_lib, q):
    eps = np.eye(6)[q]
    for x in ([5000.0, -4000.0, 0.0], [-2500.0, 3000.0, 0.0]):
        s = _sv(oracle_lib, x, [0.0, 0.0, 2000.0], 3000.0, 2000.0, 1500.0, 0.3, eps)
        ref = _sv(oracle_lib, [x[0], x[1], 1500.0], [0.0, 0.0, 2000.0], 3000.0, 2000.0, 1500.0, 0.3, eps)
        assert np.max(np.abs(s[[2, 4, 5]])) < 2e-8 * np.max(np.abs(ref))


@pytest.mark.parametrize("axis", ["L", "T", "W"])
def test_bml17_cuboid_additivity(oracle_lib, axis):
    """A cuboid split in two halves produces the sum of their fields."""
    q = np.array([1000.0, -500.0, 2000.0])
    L, T, W, th = 3000.0, 2000.0, 1500.0, 0.4
    sv = np.array([np.cos(th), np.sin(th), 0.0])
    nv = np.array([-np.sin(th), np.cos(th), 0.0])
    if axis == "L":
        halves = [(q, L / 2, T, W), (q + sv * L / 2, L / 2, T, W)]
    elif axis == "T":
        halves = [(q - nv * T / 4, L, T / 2, W), (q + nv * T / 4, L, T / 2, W)]
    else:
        halves = [(q, L, T, W / 2), (q + np.array([0, 0, W / 2]), L, T, W / 2)]
    rng = np.random.default_rng(9)
    for _ in range(4):
        x = rng.uniform([-4e3, -4e3, 4500.0], [6e3, 5e3, 7e3])
        for k in range(6):
            eps = np.eye(6)[k]
            whole = _sv(oracle_lib, x, q, L, T, W, th, eps)
            parts = sum(_sv(oracle_lib, x, qq, LL, TT, WW, th, eps) for qq, LL, TT, WW in halves)
            assert np.max(np.abs(whole - parts)) < 3e-8 * np.max(np.abs(whole))   # numerical derivative


def test_bml17_thin_layer_is_a_dislocation(oracle_lib):
    """A thin vertical layer of thickness T with shear eigenstrain e12 radiates
    like a vertical strike-slip fault with slip 2 e12 T (Okada restatement) up
    to O(T / distance)."""
    q = np.array([0.0, 0.0, 1000.0])
    L, W, T = 4000.0, 3000.0, 2.0
    e12 = 1.0e-3
    x = np.array([2500.0, 3500.0, 2500.0])
    # cuboid: strike 0, centred on the plane x2 = 0 (q is the strike-line corner)
    s_vol = _sv(oracle_lib, x, q, L, T, W, 0.0, np.array([0, e12, 0, 0, 0, 0.0]))
    s_ok = oracle_lib.okada_stress(0, x, q, L, W, 0.0, np.pi / 2, 2 * e12 * T, 0.0, 0.0, MU, 30.0e3)
    assert np.max(np.abs(s_vol - s_ok)) < 5e-3 * np.max(np.abs(s_ok))


def test_cfg2_rake_is_oblique_and_marches(oracle_lib):
    """The megathrust configuration slips at an oblique rake: at exactly 90 deg
    its strike components are rounding residue and the main loop's relative
    error norm collapses the step size (fortran/3d/src/ratestate.f90:314-315),
    at 60 deg the same 200-triangle model marches to its first event."""
    from unicycle_b200 import configs
    c = configs.cfg2(nx=10, nz=10)
    assert abs(np.degrees(c["friction"]["rake"][0]) - configs.CFG2_RAKE_DEG) < 1e-12
    i1, i2, i3, v = c["mesh"]["tri"]
    G = oracle_lib.Mesh(c["mu"], c["lam"], tri=(v, i1, i2, i3)).build_g()

    def march(rake_deg, nsteps):
        fr = dict(c["friction"])
        fr["rake"] = np.full(c["n_patch"], np.radians(rake_deg))
        md = oracle_lib.Model(G, fr)
        y, t, dt, rej = configs.steady_state(np.full(c["n_patch"], 0.9e-9), fr), 0.0, c["dt0"], 0
        for _ in range(nsteps):
            rc, t, y, _, dt, _, nr = md.step(t, y, dt, c["epsilon"])
            assert rc == 0
            rej += nr
        return t / configs.YEAR, rej

    t60, rej60 = march(configs.CFG2_RAKE_DEG, 100)
    t90, rej90 = march(90.0, 100)
    assert t60 > 1.0 and rej60 <= 5, (t60, rej60)
    assert t90 < 1e-9 and rej90 > 100, (t90, rej90)


# ---- Mindlin's point force and the independent cuboid route -----------------

def _lame(mu, nu):
    return 2.0 * mu * nu / (1.0 - 2.0 * nu)


def test_mindlin_green_function(oracle_lib):
    """Mindlin's half-space Green's function (oracle/mindlin.cc): Navier's
    equations away from the source, a traction-free surface, the Kelvin
    singularity at the source, and reciprocity G_ij(x; xi) = G_ji(xi; x)."""
    G0, nu = 30.0e3, 0.25
    lam = _lame(G0, nu)
    c = 900.0

    def u(p, cc=c):
        return oracle_lib.mindlin(p[0], p[1], p[2], cc, G0, nu)

    h = 0.5

    def grad(p):
        g = np.zeros((3, 3, 3))                       # g[i, j, d] = d u_ij / d x_d
        for d in range(3):
            e = np.zeros(3)
            e[d] = h
            g[:, :, d] = (8 * (u(p + e) - u(p - e)) - (u(p + 2 * e) - u(p - 2 * e))) / (12 * h)
        return g

    def stress(p):
        g = grad(p)
        s = np.zeros((3, 3, 3))                       # s[j][a, b]: force along j
        for j in range(3):
            eps = 0.5 * (g[:, j, :] + g[:, j, :].T)
            s[j] = lam * np.trace(eps) * np.eye(3) + 2 * G0 * eps
        return s

    rng = np.random.default_rng(4)
    for _ in range(5):
        p = np.array([rng.uniform(-2e3, 2e3), rng.uniform(-2e3, 2e3), rng.uniform(200.0, 3e3)])
        if np.linalg.norm(p - [0, 0, c]) < 300.0:
            continue
        # div(stress) = 0: second differences of the stress
        hh = 2.0
        div = np.zeros((3, 3))
        for d in range(3):
            e = np.zeros(3)
            e[d] = hh
            div += ((stress(p + e) - stress(p - e)) / (2 * hh))[:, :, d]
        scale = np.max(np.abs(stress(p))) / np.linalg.norm(p - [0, 0, c])
        assert np.max(np.abs(div)) < 1e-5 * scale
    # traction-free surface: sigma_i3 = 0 at z = 0 (one-sided stencil in z)
    for _ in range(4):
        p = np.array([rng.uniform(-3e3, 3e3), rng.uniform(-3e3, 3e3), 0.0])
        g = np.zeros((3, 3, 3))
        for d in range(2):
            e = np.zeros(3)
            e[d] = h
            g[:, :, d] = (8 * (u(p + e) - u(p - e)) - (u(p + 2 * e) - u(p - 2 * e))) / (12 * h)
        f = [u(p + np.array([0, 0, k * h])) for k in range(5)]
        g[:, :, 2] = (-25 * f[0] + 48 * f[1] - 36 * f[2] + 16 * f[3] - 3 * f[4]) / (12 * h)
        for j in range(3):
            eps = 0.5 * (g[:, j, :] + g[:, j, :].T)
            s = lam * np.trace(eps) * np.eye(3) + 2 * G0 * eps
            assert np.max(np.abs(s[:, 2])) < 1e-8 * np.max(np.abs(s)) + 1e-14
    # Kelvin singularity: G - Kelvin stays bounded at the source
    A = 1.0 / (16.0 * np.pi * G0 * (1.0 - nu))
    rest = []
    for r in (1e-1, 1e-3):
        d = np.array([0.3, -0.5, 0.81]) / np.linalg.norm([0.3, -0.5, 0.81]) * r
        kel = A * ((3 - 4 * nu) * np.eye(3) / r + np.outer(d, d) / r ** 3)
        rest.append(u(np.array([0, 0, c]) + d) - kel)
        assert np.max(np.abs(rest[-1])) < 10.0 * A / c      # the image part is O(1 / depth)
    assert np.max(np.abs(rest[0] - rest[1])) < 1e-3 * np.max(np.abs(rest[1]))
    # reciprocity: u_ij(x; xi) = u_ji(xi; x)
    for _ in range(5):
        x = rng.uniform([-2e3, -2e3, 100.0], [2e3, 2e3, 3e3])
        xi = rng.uniform([-2e3, -2e3, 100.0], [2e3, 2e3, 3e3])
        a = oracle_lib.mindlin(x[0] - xi[0], x[1] - xi[1], x[2], xi[2], G0, nu)
        b = oracle_lib.mindlin(xi[0] - x[0], xi[1] - x[1], xi[2], x[2], G0, nu)
        assert np.max(np.abs(a - b.T)) < 1e-12 * np.max(np.abs(a))


@pytest.mark.parametrize("region", ["inside", "near", "far", "surface"])
def test_bml17_closed_forms_match_mindlin_route(oracle_lib, region):
    """The Barbot et al. closed forms (numerically differentiated, x87) against
    the independent Mindlin route (point force over the faces, exact
    derivatives): every eigenstrain component, receivers inside the cuboid,
    next to it (within 0.3 of its size of a face), far from it and on the free
    surface.  Measured: 8e-11 inside, 1e-8 near, 7e-11 far, 2e-11 surface."""
    q = np.array([1000.0, -500.0, 3000.0])
    L, T, W, th = 2000.0, 1500.0, 1800.0, 0.3
    ct, st = np.cos(th), np.sin(th)
    rng = np.random.default_rng({"inside": 1, "near": 2, "far": 3, "surface": 4}[region])
    tol = {"inside": 1e-9, "near": 5e-8, "far": 1e-9, "surface": 1e-9}[region]
    for _ in range(6):
        if region == "inside":
            f = (rng.uniform(0.1 * L, 0.9 * L), rng.uniform(-0.4 * T, 0.4 * T), rng.uniform(q[2] + 0.1 * W, q[2] + 0.9 * W))
        elif region == "near":
            f = (rng.uniform(-0.3 * L, 1.3 * L), rng.choice([-1, 1]) * rng.uniform(0.55 * T, 0.8 * T),
                 rng.uniform(q[2] - 0.3 * W, q[2] + 1.3 * W))
        elif region == "far":
            f = (rng.uniform(-5 * L, 6 * L), rng.uniform(-5 * T, 5 * T), rng.uniform(0.0, q[2] + 5 * W))
        else:
            f = (rng.uniform(-3 * L, 4 * L), rng.uniform(-3 * T, 3 * T), 0.0)
        x = np.array([q[0] + f[0] * ct - f[1] * st, q[1] + f[0] * st + f[1] * ct, f[2]])
        for k in range(6):
            eps = np.eye(6)[k] * 1e-6
            a = oracle_lib.bml17_stress(x, q, L, T, W, th, eps, MU, NU)
            b = oracle_lib.bml17_stress_mindlin(x, q, L, T, W, th, eps, MU, NU)
            assert np.max(np.abs(a - b)) <= tol * np.max(np.abs(b)), (region, k, a, b)
