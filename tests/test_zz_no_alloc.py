"""The allocation-free entry point ucg_odefun_noalloc, for callers that cannot
allocate device memory when they evaluate the right-hand side (their device
memory belongs to another allocator, or they run a loop that must never call
cudaMalloc): its result must equal the context-based ucg_odefun on the same
inputs, on two calls in a row (the second call reuses the fixed scratch array
the first one left behind), free device memory must not change across a call,
and its refusals and device-side status must behave as documented.

Collected last (file name) so that a failure here stops a `-x` run only after
every other test has run; it also passes alone in a fresh process.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UCG_OK, UCG_E_BADARG, UCG_E_NONFINITE = 0, 1, 5


def _model(ucg):
    import torch
    from unicycle_b200 import configs

    c = configs.cfg1(nx=16, nz=8)
    sim = ucg.Simulation(c["mu"], c["lam"])
    configs.build(sim, c)
    fr = c["friction"]
    dev = torch.device("cuda:0")
    K = torch.from_numpy(sim.copy_G()).to(dev)             # caller-owned device matrix
    params = [torch.from_numpy(np.ascontiguousarray(p, dtype=np.float64)).to(dev) for p in (
        fr["Vpl"] * np.cos(fr["rake"]), fr["Vpl"] * np.sin(fr["rake"]), fr["a"], fr["b"], fr["sig"],
        fr["L"], fr["damping"])]
    return c, sim, K, params


def test_noalloc_odefun_matches_context_odefun(ucg):
    import torch

    c, sim, K, params = _model(ucg)
    n_p = c["n_patch"]
    dev = K.device
    lib = ucg.load()
    rng = np.random.default_rng(3)
    stream = torch.cuda.current_stream(dev)
    status = torch.full((1,), -1, dtype=torch.int32, device=dev)
    ys = []
    for call in range(2):
        y = c["y0"].copy()
        y[6::7] += rng.normal(0, 0.5, n_p)
        y[5::7] += rng.normal(0, 0.2, n_p)
        ys.append(y)
    want = [sim.odefun(y)[0] for y in ys]
    yd = [torch.from_numpy(y).to(dev) for y in ys]
    out = torch.full((7 * n_p,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    for call in range(2):
        status.fill_(-1)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(dev)[0]
        st = lib.ucg_odefun_noalloc(K.data_ptr(), 2 * n_p, 3 * n_p, n_p, yd[call].data_ptr(),
                                    *[p.data_ptr() for p in params], out.data_ptr(), stream.cuda_stream,
                                    status.data_ptr())
        assert st == UCG_OK, st
        stream.synchronize()
        free1 = torch.cuda.mem_get_info(dev)[0]
        if call == 1:
            # the first call may load the library's device code; the second allocates nothing
            assert free1 == free0, (free0, free1)
        assert int(status.item()) == UCG_OK
        got = out.cpu().numpy()
        scale = np.maximum(np.abs(want[call]).reshape(n_p, 7).max(axis=0), 1e-300)
        err = np.abs(got - want[call]).reshape(n_p, 7) / scale
        assert np.all(np.isfinite(got))
        assert err.max() < 1e-10, (call, err.max(axis=0))

    # the default (NULL) stream, no status word: same result
    out.fill_(float("nan"))
    torch.cuda.synchronize()
    assert lib.ucg_odefun_noalloc(K.data_ptr(), 2 * n_p, 3 * n_p, n_p, yd[1].data_ptr(),
                                  *[p.data_ptr() for p in params], out.data_ptr(), None, None) == UCG_OK
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    scale = np.maximum(np.abs(want[1]).reshape(n_p, 7).max(axis=0), 1e-300)
    assert (np.abs(got - want[1]).reshape(n_p, 7) / scale).max() < 1e-10
    sim.close()


def test_noalloc_refusals_and_status(ucg):
    import torch

    c, sim, K, params = _model(ucg)
    sim.close()
    n_p = c["n_patch"]
    dev = K.device
    lib = ucg.load()
    stream = torch.cuda.current_stream(dev)
    y = torch.from_numpy(c["y0"].copy()).to(dev)
    out = torch.zeros(7 * n_p, dtype=torch.float64, device=dev)
    status = torch.full((1,), -1, dtype=torch.int32, device=dev)
    pp = [p.data_ptr() for p in params]

    def call(Kp, n, m, np_, yp):
        return lib.ucg_odefun_noalloc(Kp, n, m, np_, yp, *pp, out.data_ptr(), stream.cuda_stream,
                                      status.data_ptr())

    # refused on the host before anything is queued (the status word stays -1)
    big = (1 << 20) + 1
    assert call(K.data_ptr(), 2 * big, 3 * big, big, y.data_ptr()) == UCG_E_BADARG   # beyond the scratch
    assert call(K.data_ptr(), 2 * n_p + 2, 3 * n_p, n_p, y.data_ptr()) == UCG_E_BADARG  # n != 2 np
    assert call(K.data_ptr(), 2 * n_p, 3 * n_p + 3, n_p, y.data_ptr()) == UCG_E_BADARG  # m != 3 np
    assert call(K.data_ptr() + 8, 2 * n_p, 3 * n_p, n_p, y.data_ptr()) == UCG_E_BADARG  # K off 16 B
    assert call(K.data_ptr(), 2 * n_p, 3 * n_p, n_p, y.data_ptr() + 4) == UCG_E_BADARG  # y off 8 B
    assert call(0, 2 * n_p, 3 * n_p, n_p, y.data_ptr()) == UCG_E_BADARG
    torch.cuda.synchronize()
    assert int(status.item()) == -1

    # a non-finite state is reported through the status word
    yb = c["y0"].copy()
    yb[6 + 7 * 5] = float("nan")
    ybd = torch.from_numpy(yb).to(dev)
    assert call(K.data_ptr(), 2 * n_p, 3 * n_p, n_p, ybd.data_ptr()) == UCG_OK
    stream.synchronize()
    assert int(status.item()) == UCG_E_NONFINITE
    # and the next clean call reports UCG_OK again (the control block is reset per call)
    assert call(K.data_ptr(), 2 * n_p, 3 * n_p, n_p, y.data_ptr()) == UCG_OK
    stream.synchronize()
    assert int(status.item()) == UCG_OK
    assert np.all(np.isfinite(out.cpu().numpy()))
