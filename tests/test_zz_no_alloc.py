"""The allocation-free entry point ucg_odefun_noalloc, for callers that cannot
allocate device memory when they evaluate the right-hand side: its result must
equal the context-based ucg_odefun on the same inputs, on two calls in a row
(the second call reuses the fixed scratch array the first one left behind).

Collected last (file name) so that a failure here stops a `-x` run only after
every other test has run; it also passes alone in a fresh process.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_odefun_matches_context_odefun(ucg):
    import torch
    from unicycle_b200 import configs

    c = configs.cfg1(nx=16, nz=8)
    n_p = c["n_patch"]
    sim = ucg.Simulation(c["mu"], c["lam"])
    configs.build(sim, c)
    fr = c["friction"]
    dev = torch.device("cuda:0")
    K = torch.from_numpy(sim.copy_G()).to(dev)             # caller-owned device matrix
    params = [torch.from_numpy(np.ascontiguousarray(p, dtype=np.float64)).to(dev) for p in (
        fr["Vpl"] * np.cos(fr["rake"]), fr["Vpl"] * np.sin(fr["rake"]), fr["a"], fr["b"], fr["sig"],
        fr["L"], fr["damping"])]
    lib = ucg.load()
    rng = np.random.default_rng(3)
    torch.cuda.synchronize()
    for call in range(2):
        y = c["y0"].copy()
        y[6::7] += rng.normal(0, 0.5, n_p)
        y[5::7] += rng.normal(0, 0.2, n_p)
        want, _ = sim.odefun(y)
        yd = torch.from_numpy(y).to(dev)
        out = torch.full((7 * n_p,), float("nan"), dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev)
        st = lib.ucg_odefun_noalloc(K.data_ptr(), 2 * n_p, 3 * n_p, n_p, yd.data_ptr(),
                                    *[p.data_ptr() for p in params], out.data_ptr(), stream.cuda_stream)
        assert st == 0, st
        stream.synchronize()
        got = out.cpu().numpy()
        scale = np.maximum(np.abs(want).reshape(n_p, 7).max(axis=0), 1e-300)
        err = np.abs(got - want).reshape(n_p, 7) / scale
        assert np.all(np.isfinite(got))
        assert err.max() < 1e-10, (call, err.max(axis=0))
    # sizes beyond the fixed scratch are refused without touching the device
    assert lib.ucg_odefun_noalloc(K.data_ptr(), 2 * (1 << 20) + 2, 3 * ((1 << 20) + 1), (1 << 20) + 1,
                                  yd.data_ptr(), *[p.data_ptr() for p in params], out.data_ptr(),
                                  stream.cuda_stream) == 1
    sim.close()
