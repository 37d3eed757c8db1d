"""Generate golden fixtures from the reference's own Nikkhoo-Walter C routine.

The reference sources fortran/3d/src/StrainInHalfSpace.c and DispInHalfSpace.c
are compiled unchanged into oracle/_ref/libnw15ref.so (oracle/Makefile, target
`ref`); this script calls straininhalfspace_ exactly as computeStressNikkhoo15
does (fortran/3d/src/nikkhoo15.f90:120-163) and writes:

  nw15_pairs.npz   stress (NED s11..s33) for seeded random triangle/point pairs,
                   unit strike and unit dip slip
  nw15_mesh_G.npz  the full interaction matrix in the reference layout
                   (greens.f90:176-218 traction rows) for a 6 x 5 (60-triangle)
                   curved-megathrust mesh from unicycle_b200.configs.cfg2
  nw15_disp_pairs.npz  displacement (north, east, down) from dispinhalfspace_
                   called as computeDisplacementNikkhoo15 does
                   (nikkhoo15.f90:324-367), seeded triangle/point pairs with
                   surface-reaching triangles and surface points, unit strike
                   and unit dip slip

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from unicycle_b200 import configs  # noqa: E402

MU = 30.0e3
LAM = 30.0e3


def traction(sv, dv, nv, s):
    """fortran/3d/src/nikkhoo15.f90:208-220"""
    s11, s12, s13, s22, s23, s33 = s
    a = nv[0] * s11 + nv[1] * s12 + nv[2] * s13
    b = nv[0] * s12 + nv[1] * s22 + nv[2] * s23
    c = nv[0] * s13 + nv[1] * s23 + nv[2] * s33
    return np.array([a * sv[0] + b * sv[1] + c * sv[2], a * dv[0] + b * dv[1] + c * dv[2],
                     a * nv[0] + b * nv[1] + c * nv[2]])


def pairs(n=300, seed=11):
    rng = np.random.default_rng(seed)
    P = rng.uniform([-5e3, -5e3, 0.0], [5e3, 5e3, 8e3], size=(n, 3, 3))
    P[: n // 10, :, 2] = np.maximum(P[: n // 10, :, 2] - 8e3, 0.0)   # some surface-reaching TDs
    X = rng.uniform([-10e3, -10e3, 0.0], [10e3, 10e3, 12e3], size=(n, 3))
    S = np.zeros((n, 2, 6))
    for k in range(n):
        for j, (s, d) in enumerate(((1.0, 0.0), (0.0, 1.0))):
            S[k, j] = oracle.nw15_stress_ref(X[k], P[k, 0], P[k, 1], P[k, 2], s, d, 0.0, MU, LAM)
    return P, X, S


def disp_pairs(n=200, seed=13):
    rng = np.random.default_rng(seed)
    P = rng.uniform([-5e3, -5e3, 0.0], [5e3, 5e3, 8e3], size=(n, 3, 3))
    P[: n // 10, :, 2] = np.maximum(P[: n // 10, :, 2] - 8e3, 0.0)
    X = rng.uniform([-10e3, -10e3, 0.0], [10e3, 10e3, 12e3], size=(n, 3))
    X[n // 2:, 2] = 0.0   # half of the points on the free surface (GPS-like)
    U = np.zeros((n, 2, 3))
    for k in range(n):
        for j, (s, d) in enumerate(((1.0, 0.0), (0.0, 1.0))):
            U[k, j] = oracle.nw15_disp_ref(X[k], P[k, 0], P[k, 1], P[k, 2], s, d, 0.0, MU, LAM)
    return P, X, U


def mesh_G(nx=6, nz=5):
    c = configs.cfg2(nx=nx, nz=nz)
    i1, i2, i3, v = c["mesh"]["tri"]
    M = oracle.Mesh(MU, LAM, tri=(v, i1, i2, i3))
    sv, dv, nv, xc = M.tri_frames
    n = len(i1)
    G = np.zeros((3 * n, 2 * n))
    for r in range(n):
        for s in range(n):
            A, B, C = v[i1[s] - 1], v[i2[s] - 1], v[i3[s] - 1]
            for j, (ss, ds) in enumerate(((1.0, 0.0), (0.0, 1.0))):
                st = oracle.nw15_stress_ref(xc[r], A, B, C, ss, ds, 0.0, MU, LAM)
                G[3 * r: 3 * r + 3, 2 * s + j] = traction(sv[r], dv[r], nv[r], st)
    return (i1, i2, i3, v), G


def main():
    oracle.build(ref=True)
    if oracle.ref_lib() is None:
        raise SystemExit("reference C not available (oracle/_ref not built)")
    P, X, S = pairs()
    np.savez_compressed(os.path.join(HERE, "nw15_pairs.npz"), P=P, X=X, S=S, mu=MU, lam=LAM)
    (i1, i2, i3, v), G = mesh_G()
    np.savez_compressed(os.path.join(HERE, "nw15_mesh_G.npz"), i1=i1, i2=i2, i3=i3, v=v, G=G, mu=MU, lam=LAM)
    P, X, U = disp_pairs()
    np.savez_compressed(os.path.join(HERE, "nw15_disp_pairs.npz"), P=P, X=X, U=U, mu=MU, lam=LAM)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
