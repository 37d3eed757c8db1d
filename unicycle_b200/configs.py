"""Seeded synthetic workloads of the 3-D quasi-dynamic benchmark configurations.

Units: lengths in m, stresses in MPa, time in s, angles in radians.
Every generator returns plain numpy dictionaries:
  mesh:     {"rect": (x, L, W, strike, dip)} and/or {"tri": (i1, i2, i3, v)}
  friction: per patch Vpl, rake, mu0, sig, a, b, L, Vo, damping
  y0:       initial state vector (7 per patch)
plus the elastic moduli and integration settings.  Values the benchmark
descriptions leave open (mu0 = 0.6, Vo = 1e-6 m/s, 1 yr = 3.15576e7 s, the
megathrust bottom depth) are fixed here and recorded in the returned dict.
"""
import numpy as np

YEAR = 3.15576e7
MU = 30.0e3          # MPa
NU = 0.25
LAM = 2.0 * MU * NU / (1.0 - 2.0 * NU)   # = MU for nu = 1/4
VS = 3464.0          # m/s
ETA = MU / (2.0 * VS)  # MPa s / m (radiation damping)
MU0 = 0.6
VO = 1.0e-6
LG10 = np.log(10.0)


def steady_state(V0, fr):
    """Initial state at steady state theta = L/V0, traction along the rake
    (fortran/3d/src/ratestate.f90:589-607 with V0 in place of 0.99 Vpl)."""
    n = len(V0)
    y = np.zeros(7 * n)
    tau = fr["sig"] * (fr["mu0"] + (fr["a"] - fr["b"]) * np.log(V0 / fr["Vo"])) - fr["damping"] * V0
    y[2::7] = tau * np.cos(fr["rake"])
    y[3::7] = tau * np.sin(fr["rake"])
    y[5::7] = np.log(fr["L"] / V0) / LG10
    y[6::7] = np.log(V0) / LG10
    return y


def cfg1(nx=32, nz=16, size=1250.0, seed=1):
    """Vertical strike-slip fault, nx x nz Okada rectangles of `size` m, a central
    velocity-weakening zone (columns 5-28, rows 5-12 of 32 x 16), V0 = 0.9 Vpl
    lognormal(0, 0.1), rtol 1e-8, 300 yr."""
    ix, iz = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    ix, iz = ix.ravel(), iz.ravel()
    n = nx * nz
    x = np.stack([ix * size, np.zeros(n), iz * size], axis=1).astype(float)
    L = np.full(n, size)
    W = np.full(n, size)
    strike = np.zeros(n)
    dip = np.full(n, np.pi / 2)
    # velocity-weakening window scaled from the 32 x 16 layout
    c0, c1 = int(round(4 * nx / 32)), int(round(28 * nx / 32))
    r0, r1 = int(round(4 * nz / 16)), int(round(12 * nz / 16))
    vw = (ix >= c0) & (ix < c1) & (iz >= r0) & (iz < r1)
    fr = dict(Vpl=np.full(n, 1.0e-9), rake=np.zeros(n), mu0=np.full(n, MU0), sig=np.full(n, 50.0),
              a=np.full(n, 0.01), b=np.where(vw, 0.014, 0.006), L=np.full(n, 0.01), Vo=np.full(n, VO),
              damping=np.full(n, ETA))
    rng = np.random.default_rng(seed)
    V0 = 0.9 * fr["Vpl"] * np.exp(0.1 * rng.standard_normal(n))
    return dict(name=f"cfg1-strike-slip-{nx}x{nz}", mu=MU, lam=LAM, mesh=dict(rect=(x, L, W, strike, dip)),
                friction=fr, y0=steady_state(V0, fr), epsilon=1.0e-8, t_end=300 * YEAR, dt0=1.0e-3,
                n_patch=n)


def tilt(cfg, dip_deg=70.0, rake_deg=30.0):
    """A rectangle-fault config tilted to `dip_deg` with every rake set to
    `rake_deg` and the initial state recomputed at the same velocities: no
    state component is zero by symmetry, so the main loop's relative error
    norm acts on physical values only (a vertical fault slipping at rake 0 has
    dip slip and dip traction that are rounding residue).  Modifies and
    returns cfg."""
    x, L, W, st, dp = cfg["mesh"]["rect"]
    cfg["mesh"]["rect"] = (x, L, W, st, np.full_like(dp, np.radians(dip_deg)))
    fr = cfg["friction"]
    fr["rake"] = np.full_like(fr["rake"], np.radians(rake_deg))
    cfg["y0"] = steady_state(np.exp(cfg["y0"][6::7] * LG10), fr)
    return cfg


def megathrust_mesh(nx=100, nz=100, dx=2000.0, z_bottom=50.0e3):
    """Curved thrust surface: strike north, dipping east; dip 10 deg at the trench
    rising linearly to 25 deg at 40 km depth, constant below; bottom edge at
    z_bottom.  nx along-strike cells of dx, nz down-dip rows of equal down-dip
    length; every quad split into 2 triangles."""
    # profile: integrate dz/ds = sin(dip(z)), dx/ds = cos(dip(z)) to z_bottom
    def dip_at(z):
        return np.radians(10.0 + 15.0 * np.clip(z / 40.0e3, 0.0, 1.0))
    ds = 1.0
    s_pts, e_pts, z_pts = [0.0], [0.0], [0.0]
    while z_pts[-1] < z_bottom:
        d = dip_at(z_pts[-1] + 0.5 * ds * np.sin(dip_at(z_pts[-1])))
        e_pts.append(e_pts[-1] + ds * np.cos(d))
        z_pts.append(z_pts[-1] + ds * np.sin(d))
        s_pts.append(s_pts[-1] + ds)
    s_pts, e_pts, z_pts = map(np.asarray, (s_pts, e_pts, z_pts))
    s_tot = np.interp(z_bottom, z_pts, s_pts)
    s_nodes = np.linspace(0.0, s_tot, nz + 1)
    e_nodes = np.interp(s_nodes, s_pts, e_pts)
    z_nodes = np.interp(s_nodes, s_pts, z_pts)
    n_nodes = np.arange(nx + 1) * dx
    N, K = np.meshgrid(n_nodes, np.arange(nz + 1), indexing="ij")
    v = np.stack([N.ravel(), e_nodes[K.ravel()], z_nodes[K.ravel()]], axis=1)
    vid = lambda i, k: i * (nz + 1) + k + 1   # 1-based
    i1, i2, i3 = [], [], []
    for i in range(nx):
        for k in range(nz):
            a, b, c, d = vid(i, k), vid(i + 1, k), vid(i + 1, k + 1), vid(i, k + 1)
            i1 += [a, a]
            i2 += [b, c]
            i3 += [c, d]
    return np.array(i1), np.array(i2), np.array(i3), v


def tri_centroids(i1, i2, i3, v):
    return (v[i1 - 1] + v[i2 - 1] + v[i3 - 1]) / 3.0


CFG2_RAKE_DEG = 60.0


def cfg2(nx=100, nz=100, seed=2, rake_deg=CFG2_RAKE_DEG):
    """Curved megathrust, Nikkhoo-Walter triangles (2 nx nz of them), oblique
    rake (60 deg: convergence with a left-lateral strike component), a = 0.01
    with depth-dependent a-b, Dc log-uniform [5, 50] mm,
    sigma = min(18 MPa/km * z, 50 MPa), 1000 yr.

    The rake is oblique on purpose.  At exactly 90 deg the strike components
    of the state (strike slip, strike traction) are rounding residue
    (Vpl cos(pi/2) = 6e-17 Vpl), and the relative error norm of the main loop
    (yscal = |y| + |h dydt| + 1e-30, fortran/3d/src/ratestate.f90:314-315) acts
    on that residue: the step size collapses to 1e-9..1e-5 s and a 200-triangle
    model covers 7e-11 yr in 4,000 steps, while at 60 deg the same model
    reaches its first event at 2.76 yr with one rejected attempt."""
    i1, i2, i3, v = megathrust_mesh(nx, nz)
    n = len(i1)
    zc = tri_centroids(i1, i2, i3, v)[:, 2] / 1.0e3   # km
    amb = np.interp(zc, [0.0, 5.0, 10.0, 35.0, 40.0, 1.0e9], [0.004, 0.004, -0.004, -0.004, 0.004, 0.004])
    a = np.full(n, 0.01)
    rng = np.random.default_rng(seed)
    Dc = np.exp(rng.uniform(np.log(5.0e-3), np.log(50.0e-3), n))
    sig = np.minimum(18.0 * zc, 50.0)
    fr = dict(Vpl=np.full(n, 1.0e-9), rake=np.full(n, np.radians(rake_deg)), mu0=np.full(n, MU0), sig=sig, a=a,
              b=a - amb, L=Dc, Vo=np.full(n, VO), damping=np.full(n, ETA))
    V0 = 0.9 * fr["Vpl"]
    return dict(name=f"cfg2-megathrust-{n}tri", mu=MU, lam=LAM, mesh=dict(tri=(i1, i2, i3, v)), friction=fr,
                y0=steady_state(np.full(n, V0[0]), fr), epsilon=1.0e-8, t_end=1000 * YEAR, dt0=1.0e-3,
                n_patch=n, z_bottom=50.0e3)


def build(sim, cfg, okada_mode=0):
    """Load a config into a Simulation and assemble its Green's functions."""
    m = cfg["mesh"]
    if "rect" in m:
        sim.set_rectangles(*m["rect"])
    if "tri" in m:
        sim.set_triangles(*m["tri"])
    fr = cfg["friction"]
    sim.set_friction(fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"],
                     fr["damping"])
    sim.set_tolerance(cfg["epsilon"])
    sim.buildG(okada_mode)
    return sim


def cfg3(nxf=64, nzf=64, nxv=32, nyv=16, nzv=16, cell=2000.0, seed=3):
    """Coupled fault and distributed deformation: a vertical strike-slip fault of
    nxf x nzf Okada rectangles (64 km x 30 km at full size) above a mantle wedge
    of nxv x nyv x nzv vertical cuboids of `cell` m starting at 30 km (16 layers of
    2 km reach 62 km), linear Maxwell rheology (npowerm = 1,
    gammadot0m = 1/(2 eta)), viscosity log-uniform in [1e18, 1e20] Pa s, no
    background strain rate.  The initial state is the response to a uniform 5 m
    strike slip on the fault (one product with the fault columns of K); 50 yr."""
    dx, dz = 64.0e3 / nxf, 30.0e3 / nzf
    ix, iz = np.meshgrid(np.arange(nxf), np.arange(nzf), indexing="ij")
    ix, iz = ix.ravel(), iz.ravel()
    nf = nxf * nzf
    x = np.stack([ix * dx, np.zeros(nf), iz * dz], axis=1).astype(float)
    rect = (x, np.full(nf, dx), np.full(nf, dz), np.zeros(nf), np.full(nf, np.pi / 2))
    # cuboids under the fault: x along strike, y across, z from 30 km.  One
    # column of cuboids is centred on the fault plane (y = 0), so that no fault
    # receiver lies on the plane of a cuboid face: there the closed-form
    # integrals (the reference's derivative forms too, e.g. the 0/0 of
    # y1**2/(y1**2+(x2p-y2)**2) at strainvolume.f90:1860) are undefined.
    jx, jy, jz = np.meshgrid(np.arange(nxv), np.arange(nyv), np.arange(nzv), indexing="ij")
    jx, jy, jz = jx.ravel(), jy.ravel(), jz.ravel()
    nv = nxv * nyv * nzv
    x0 = 32.0e3 - nxv * cell / 2.0
    vx = np.stack([x0 + jx * cell, (jy - nyv // 2) * cell, 30.0e3 + jz * cell], axis=1)
    vol = (vx, np.full(nv, cell), np.full(nv, cell), np.full(nv, cell), np.zeros(nv))
    fr = dict(Vpl=np.full(nf, 1.0e-9), rake=np.zeros(nf), mu0=np.full(nf, MU0), sig=np.full(nf, 50.0),
              a=np.full(nf, 0.01), b=np.full(nf, 0.006), L=np.full(nf, 0.01), Vo=np.full(nf, VO),
              damping=np.full(nf, ETA))
    rng = np.random.default_rng(seed)
    eta = np.exp(rng.uniform(np.log(1.0e18), np.log(1.0e20), nv)) / 1.0e6   # MPa s
    rheo = dict(ebg=np.zeros((nv, 6)), gammadot0m=1.0 / (2.0 * eta), npowerm=np.ones(nv),
                nGm=np.full(nv, MU), nQm=np.zeros(nv), nRm=np.ones(nv), To=np.ones(nv))
    y0 = np.zeros(7 * nf + 12 * nv)
    y0[:7 * nf] = steady_state(np.full(nf, 0.99e-9), fr)
    return dict(name=f"cfg3-coupled-{nf}rect-{nv}vol", mu=MU, lam=LAM,
                mesh=dict(rect=rect, vol=vol), friction=fr, rheology=rheo, y0=y0, epsilon=1.0e-8,
                t_end=50 * YEAR, dt0=1.0e-3, n_patch=nf, n_vol=nv, coseismic_slip=5.0)


def coseismic_preload(K, cfg):
    """Add the stress change of the config's uniform coseismic strike slip to the
    initial state (tractions on the fault, stresses in the volumes): one product
    of the fault-source columns of K (rows = receiver DOFs) with the slip."""
    nf, nv = cfg["n_patch"], cfg.get("n_vol", 0)
    s = np.zeros(K.shape[1])
    s[0:2 * nf:2] = cfg["coseismic_slip"]
    dt = K @ s
    y = cfg["y0"].copy()
    for c in range(3):
        y[2 + c:7 * nf:7] += dt[c:3 * nf:3]
    for c in range(6):
        y[7 * nf + 6 + c::12] += dt[3 * nf + c::6]
    return y


def build_coupled(sim, cfg):
    """Load a fault + volume config (viscous-cycles driver) and assemble."""
    sim.set_rectangles(*cfg["mesh"]["rect"])
    sim.set_volumes(*cfg["mesh"]["vol"])
    fr = cfg["friction"]
    sim.set_friction(fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"],
                     fr["damping"])
    rh = cfg["rheology"]
    sim.set_rheology(rh["ebg"], rh["gammadot0m"], rh["npowerm"], nonlinear_maxwell=True)
    sim.set_tolerance(cfg["epsilon"])
    sim.buildG()
    return sim


def cfg4(shapes=((64, 16), (64, 32), (96, 32), (128, 32)), n_sets=64, size=625.0, seed=4):
    """Batched ensemble: planar faults of nx x nz Okada rectangles of `size` m with
    seeded strike (uniform) and dip (uniform 60-90 deg), top edge at the surface;
    each with n_sets frictional parameter sets.  a = 0.01 everywhere; outside the
    velocity-weakening window (the cfg1 window scaled to nx x nz) b = 0.006 and
    Dc = 10 mm; inside it a-b ~ U[-0.006, -0.002] and Dc log-uniform [1, 20] mm,
    one draw per set.  sigma = 50 MPa, Vpl = 1e-9 m/s, rake 0; V0 = 0.9 Vpl
    lognormal(0, 0.1) per set, steady state; rtol 1e-8; 500 yr."""
    rng = np.random.default_rng(seed)
    geoms = []
    for nx, nz in shapes:
        phi = rng.uniform(0.0, 2.0 * np.pi)
        delta = np.radians(rng.uniform(60.0, 90.0))
        sv = np.array([np.cos(phi), np.sin(phi), 0.0])
        dv = np.array([np.sin(phi) * np.cos(delta), -np.cos(phi) * np.cos(delta), -np.sin(delta)])  # up-dip
        ix, iz = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
        ix, iz = ix.ravel(), iz.ravel()
        n = nx * nz
        x = ix[:, None] * size * sv[None, :] - iz[:, None] * size * dv[None, :]
        x[:, 2] = np.abs(x[:, 2])   # down is positive; exact zero at the top row
        mesh = dict(rect=(x, np.full(n, size), np.full(n, size), np.full(n, phi), np.full(n, delta)))
        c0, c1 = int(round(4 * nx / 32)), int(round(28 * nx / 32))
        r0, r1 = int(round(4 * nz / 16)), int(round(12 * nz / 16))
        vw = (ix >= c0) & (ix < c1) & (iz >= r0) & (iz < r1)
        sets, y0s = [], []
        for _ in range(n_sets):
            amb = rng.uniform(-0.006, -0.002)
            dc = np.exp(rng.uniform(np.log(1.0e-3), np.log(20.0e-3)))
            fr = dict(Vpl=np.full(n, 1.0e-9), rake=np.zeros(n), mu0=np.full(n, MU0), sig=np.full(n, 50.0),
                      a=np.full(n, 0.01), b=np.where(vw, 0.01 - amb, 0.006), L=np.where(vw, dc, 0.01),
                      Vo=np.full(n, VO), damping=np.full(n, ETA))
            V0 = 0.9 * fr["Vpl"] * np.exp(0.1 * rng.standard_normal(n))
            sets.append(fr)
            y0s.append(steady_state(V0, fr))
        geoms.append(dict(name=f"cfg4-{nx}x{nz}", mesh=mesh, friction=sets[0], sets=sets, y0s=y0s, n_patch=n,
                          mu=MU, lam=LAM, epsilon=1.0e-8))
    return dict(name="cfg4-ensemble", geoms=geoms, epsilon=1.0e-8, t_end=500 * YEAR, dt0=1.0e-3)


def build_ensemble(ens, cfg, sim_factory):
    """Assemble every geometry of an ensemble config (cfg4) with a Simulation made
    by sim_factory(mu, lam), add it to `ens` with all its parameter sets and
    initial states.  Returns the geometry indices."""
    ids = []
    for g in cfg["geoms"]:
        sim = sim_factory(g["mu"], g["lam"])
        try:
            build(sim, g)
            gi = ens.add_geometry(sim, len(g["sets"]))
        finally:
            sim.close()
        for i, (fr, y0) in enumerate(zip(g["sets"], g["y0s"])):
            ens.set_friction(gi, i, fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"],
                             fr["Vo"], fr["damping"])
            ens.set_state(gi, i, y0, 0.0, cfg["dt0"])
        ids.append(gi)
    ens.set_tolerance(cfg["epsilon"])
    return ids


def parameter_sets(cfg, n_sets, seed=1000):
    """n_sets frictional parameter sets of a single-geometry config, for an
    ensemble: set 0 is the config's own; every other set redraws Dc per element,
    log-uniform over the config's Dc range (seed + set index), keeping a, b and
    sigma, with the initial state at the config's V0 in steady state for the new
    Dc.  Returns (list of friction dicts, list of initial states)."""
    fr0 = cfg["friction"]
    lo, hi = float(np.min(fr0["L"])), float(np.max(fr0["L"]))
    n = cfg["n_patch"]
    V0 = 10.0 ** cfg["y0"][6::7]
    sets, y0s = [fr0], [cfg["y0"]]
    for k in range(1, n_sets):
        rng = np.random.default_rng(seed + k)
        fr = dict(fr0)
        fr["L"] = np.exp(rng.uniform(np.log(lo), np.log(hi), n)) if hi > lo else fr0["L"].copy()
        sets.append(fr)
        y0s.append(steady_state(V0, fr))
    return sets, y0s


def cfg1_instances(seeds, nx=32, nz=16, size=1250.0):
    """cfg1 once per seed (the seed draws the lognormal initial slip-rate
    perturbation; geometry and friction are shared): the config of seed[0] and
    the initial states of all seeds, for an ensemble."""
    cfgs = [cfg1(nx=nx, nz=nz, size=size, seed=s) for s in seeds]
    return cfgs[0], [c["y0"] for c in cfgs]
