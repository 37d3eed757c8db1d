"""CPU tests of the C-ABI library: it loads, exports every symbol that
include/ucg.h declares, and its host-side argument checks work without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "ucg.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ucg_[A-Za-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(ucg):
    lib = ucg.load()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s


def test_python_binding_covers_header(ucg):
    from unicycle_b200 import _lib
    assert set(header_symbols()) == set(_lib.SIGNATURES)


def test_strerror_and_create_without_device(ucg):
    import torch
    lib = ucg.load()
    assert lib.ucg_strerror(4) == b"stepsize underflow in RKQS"
    assert lib.ucg_strerror(0) == b"ok"
    ctx = ctypes.c_void_p()
    # invalid moduli are rejected before any device call
    assert lib.ucg_create(ctypes.byref(ctx), 0, -1.0, 1.0, 0) == 1
    assert lib.ucg_create(ctypes.byref(ctx), 0, 1.0, 1.0, 7) == 1
    if not torch.cuda.is_available():
        assert lib.ucg_create(ctypes.byref(ctx), 0, 3e4, 3e4, 0) == 9   # UCG_E_NODEVICE
        assert not ctx.value


def test_null_context_is_rejected(ucg):
    lib = ucg.load()
    assert lib.ucg_assemble(None, 0) == 1
    assert lib.ucg_state_len(None) == -1
    assert lib.ucg_launch_count(None) == -1
    lib.ucg_destroy(None)


def test_configs_shapes():
    from unicycle_b200 import configs
    c1 = configs.cfg1()
    assert c1["n_patch"] == 512 and c1["y0"].shape == (7 * 512,)
    assert int(np.sum(c1["friction"]["b"] > 0.01)) == 24 * 8
    c2 = configs.cfg2()
    i1, i2, i3, v = c2["mesh"]["tri"]
    assert len(i1) == 20000 and len(v) == 101 * 101
    zc = configs.tri_centroids(i1, i2, i3, v)[:, 2]
    assert zc.max() < 50.0e3 and zc.min() > 0.0
    assert np.isclose(v[:, 2].max(), 50.0e3)
    assert np.all(c2["friction"]["sig"] <= 50.0)
    Dc = c2["friction"]["L"]
    assert Dc.min() >= 5e-3 and Dc.max() <= 50e-3
