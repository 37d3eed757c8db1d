"""CPU pins of the oracle's displacement kernels (the output path's buildO,
greens.f90:302-462): the Nikkhoo-Walter restatement against the reference's
own dispinhalfspace_ (golden fixture and, where built, the live library), the
Okada rectangle against two reference triangles, and every kernel's
displacement gradient against its already-pinned stress through Hooke's law."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
MU = LAM = 30.0e3


def _rect_as_triangles(q, L, W, strike, dip):
    sv = np.array([np.cos(strike), np.sin(strike), 0.0])
    dv = np.array([np.sin(strike) * np.cos(dip), -np.cos(strike) * np.cos(dip), -np.sin(dip)])
    return (q, q + L * sv, q + L * sv - W * dv), (q, q + L * sv - W * dv, q - W * dv)


def _hooke_from_gradient(disp, x, h, mu, lam):
    """stress (s11, s12, s13, s22, s23, s33) from a fourth-order central
    difference of the displacement field around x"""
    J = np.zeros((3, 3))
    for k in range(3):
        e = np.zeros(3)
        e[k] = h
        J[:, k] = (8 * (disp(x + e) - disp(x - e)) - (disp(x + 2 * e) - disp(x - 2 * e))) / (12 * h)
    eps = 0.5 * (J + J.T)
    s = lam * np.trace(eps) * np.eye(3) + 2 * mu * eps
    return np.array([s[0, 0], s[0, 1], s[0, 2], s[1, 1], s[1, 2], s[2, 2]])


def test_nw15_disp_matches_reference_golden(oracle_lib):
    g = np.load(os.path.join(GOLD, "nw15_disp_pairs.npz"))
    P, X, U = g["P"], g["X"], g["U"]
    worst = 0.0
    for k in range(len(X)):
        for j, (s, d) in enumerate(((1.0, 0.0), (0.0, 1.0))):
            a = oracle_lib.nw15_disp(X[k], P[k, 0], P[k, 1], P[k, 2], s, d, 0.0, MU, LAM)
            worst = max(worst, np.max(np.abs(a - U[k, j])) / np.max(np.abs(U[k, j])))
    assert worst < 1e-9, worst


def test_nw15_disp_live_reference(oracle_lib):
    if oracle_lib.ref_lib() is None:
        pytest.skip("reference C sources not present here")
    rng = np.random.default_rng(15)
    for _ in range(50):
        P = rng.uniform([-3e3, -3e3, 0.0], [3e3, 3e3, 6e3], size=(3, 3))
        x = rng.uniform([-8e3, -8e3, 0.0], [8e3, 8e3, 10e3])
        for s, d in ((1.0, 0.0), (0.0, 1.0)):
            a = oracle_lib.nw15_disp(x, *P, s, d, 0.0, MU, LAM)
            b = oracle_lib.nw15_disp_ref(x, *P, s, d, 0.0, MU, LAM)
            assert np.max(np.abs(a - b)) <= 1e-9 * np.max(np.abs(b))


def test_okada_disp_equals_two_triangles(oracle_lib):
    """Random rectangles of dip 15-85 degrees (and exactly 90) at random points,
    surface points included.  Closer to vertical the Okada closed forms divide
    by cos^2(dip) and lose digits (89.9 degrees: 3.5e-8), the triangles do not."""
    nw = oracle_lib.nw15_disp_ref if oracle_lib.ref_lib() is not None else oracle_lib.nw15_disp
    rng = np.random.default_rng(11)
    worst = 0.0
    for trial in range(60):
        q = np.array([0.0, 0.0, rng.uniform(0.0, 3000.0)])
        L, W = rng.uniform(1000.0, 4000.0, 2)
        strike = rng.uniform(0.0, 2 * np.pi)
        dip = np.pi / 2 if trial % 10 == 0 else np.radians(rng.uniform(15.0, 85.0))
        t1, t2 = _rect_as_triangles(q, L, W, strike, dip)
        x = rng.uniform([-6e3, -6e3, 0.0], [9e3, 9e3, 9e3])
        if trial % 7 == 0:
            x[2] = 0.0
        for s, d in ((1.0, 0.0), (0.0, 1.0)):
            ok = oracle_lib.okada_disp(oracle_lib.OKADA_FP64, x, q, L, W, strike, dip, s, d, 0.0, MU, LAM)
            tr = nw(x, *t1, s, d, 0.0, MU, LAM) + nw(x, *t2, s, d, 0.0, MU, LAM)
            worst = max(worst, np.max(np.abs(ok - tr)) / np.max(np.abs(tr)))
    assert worst < 1e-9, worst


def test_okada_disp_ref32io_close_to_fp64(oracle_lib):
    q = np.array([0.0, 0.0, 1500.0])
    x = np.array([2500.0, 1200.0, 800.0])
    a = oracle_lib.okada_disp(oracle_lib.OKADA_FP64, x, q, 2000.0, 1500.0, 0.3, 1.0, 1.0, 0.0, 0.0, MU, LAM)
    b = oracle_lib.okada_disp(oracle_lib.OKADA_REF32IO, x, q, 2000.0, 1500.0, 0.3, 1.0, 1.0, 0.0, 0.0, MU, LAM)
    assert np.max(np.abs(a - b)) < 1e-5 * np.max(np.abs(a))
    # REAL*4 outputs of DC3D; the rotation to north/east is in REAL*8 (okada92.f90:288-290)
    assert np.float64(np.float32(b[2])) == b[2]


def test_okada_disp_gradient_is_its_stress(oracle_lib):
    """strike 0: the reference's stress rotation is the chain rule there"""
    q = np.array([0.0, 0.0, 2000.0])
    for dip in (np.pi / 2, np.radians(50.0)):
        for s, d in ((1.0, 0.0), (0.0, 1.0)):
            for x in ([3500.0, 1800.0, 2500.0], [-1500.0, -2500.0, 600.0]):
                x = np.array(x)
                disp = lambda p: oracle_lib.okada_disp(0, p, q, 3000.0, 2000.0, 0.0, dip, s, d, 0.0, MU, LAM)
                fd = _hooke_from_gradient(disp, x, 1.0, MU, LAM)
                st = oracle_lib.okada_stress(0, x, q, 3000.0, 2000.0, 0.0, dip, s, d, 0.0, MU, LAM)
                assert np.max(np.abs(fd - st)) < 1e-7 * np.max(np.abs(st))


def test_nw15_disp_gradient_is_its_stress(oracle_lib):
    rng = np.random.default_rng(21)
    for _ in range(6):
        P = rng.uniform([-3e3, -3e3, 500.0], [3e3, 3e3, 6e3], size=(3, 3))
        x = rng.uniform([-8e3, -8e3, 500.0], [8e3, 8e3, 10e3])
        for s, d in ((1.0, 0.0), (0.0, 1.0)):
            disp = lambda p: oracle_lib.nw15_disp(p, *P, s, d, 0.0, MU, LAM)
            fd = _hooke_from_gradient(disp, x, 1.0, MU, LAM)
            st = oracle_lib.nw15_stress(x, *P, s, d, 0.0, MU, LAM)
            assert np.max(np.abs(fd - st)) < 1e-7 * np.max(np.abs(st))


def test_bml17_disp_gradient_is_its_stress(oracle_lib):
    """outside the cuboid, where no eigenstress is subtracted"""
    nu = 0.25
    lam = 2 * MU * nu / (1 - 2 * nu)
    q = np.array([500.0, -300.0, 2000.0])
    for x in ([4500.0, 3200.0, 1200.0], [-2500.0, 1500.0, 5200.0]):
        x = np.array(x)
        for k in range(6):
            eps = np.eye(6)[k]
            disp = lambda p: oracle_lib.bml17_disp(p, q, 3000.0, 2000.0, 1500.0, 0.4, eps, MU, nu)
            fd = _hooke_from_gradient(disp, x, 1.0, MU, lam)
            st = oracle_lib.bml17_stress(x, q, 3000.0, 2000.0, 1500.0, 0.4, eps, MU, nu)
            assert np.max(np.abs(fd - st)) < 1e-6 * np.max(np.abs(st)), (x, k)


def test_build_o_columns(oracle_lib):
    """orc_build_o stacks the per-source kernels: one column per slip component
    / eigenstrain component, rows (north, east, down) per observation point."""
    rect = (np.array([[0.0, 0.0, 1000.0], [0.0, 2000.0, 1000.0]]), np.array([2000.0, 2000.0]),
            np.array([1500.0, 1500.0]), np.array([0.0, 0.0]), np.array([np.pi / 2, np.pi / 2]))
    M = oracle_lib.Mesh(MU, LAM, rect=rect)
    xo = np.array([[3000.0, 500.0, 0.0], [-1000.0, 2500.0, 0.0], [800.0, -1200.0, 0.0]])
    O = M.build_o(xo)
    assert O.shape == (9, 4)
    for k in range(3):
        for i in range(2):
            for j, (s, d) in enumerate(((1.0, 0.0), (0.0, 1.0))):
                u = oracle_lib.okada_disp(0, xo[k], rect[0][i], 2000.0, 1500.0, 0.0, np.pi / 2, s, d, 0.0, MU, LAM)
                assert np.array_equal(O[3 * k: 3 * k + 3, 2 * i + j], u)
