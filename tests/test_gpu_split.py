"""Split-BF16 matrix with anchored stages (single instance): the integrator
driven through its first earthquake matches the FP64 integrator's onset time
within 1e-4 relative and takes a comparable number of steps.  Without anchoring
the product's rounding would dominate the embedded error estimate on the
near-zero components and stall the step size."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _first_event(sim, y0, dt0, von=1.0e-3, max_steps=20000):
    t, y, dn = 0.0, y0.copy(), dt0
    n = len(y0) // 7
    rej = 0
    for k in range(max_steps):
        if 10.0 ** y.reshape(n, 7)[:, 6].max() >= von:
            return t, k, rej
        t, y, _, dn, _, nr = sim.step(t, y, dn)
        rej += nr
    return None, max_steps, rej


def test_split_bf16_event_onset_matches_fp64(ucg):
    from unicycle_b200 import configs
    cfg = configs.cfg4(shapes=((16, 8),), n_sets=4, size=1250.0, seed=11)
    g = cfg["geoms"][0]
    sim = ucg.Simulation(g["mu"], g["lam"])
    configs.build(sim, g)
    for i in (0, 2):
        fr = g["sets"][i]
        sim.set_friction(fr["Vpl"], fr["rake"], fr["mu0"], fr["sig"], fr["a"], fr["b"], fr["L"], fr["Vo"],
                         fr["damping"])
        sim.set_precision(ucg.UCG_PREC_FP64)
        t64, k64, r64 = _first_event(sim, g["y0s"][i], cfg["dt0"])
        sim.set_precision(ucg.UCG_PREC_SPLIT_BF16)
        ts, ks, rs = _first_event(sim, g["y0s"][i], cfg["dt0"])
        print(f"set {i}: fp64 onset {t64:.9e} ({k64} steps, {r64} rejected)  split {ts:.9e} ({ks} steps, "
              f"{rs} rejected)  rel {abs(ts - t64) / t64:.2e}")
        assert t64 is not None and ts is not None
        assert abs(ts - t64) <= 1e-4 * t64
        assert ks <= 1.5 * k64 + 20
    sim.close()
