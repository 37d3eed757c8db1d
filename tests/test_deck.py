"""CPU tests of the input-deck reader (ucg_deck_*, host-only C++ in libucg):
round trips of the synthetic configurations through the reference's deck
format, the list-directed reading rules of init()/getdata.f, and the
validation the reference performs while reading (ratestate.f90:958-1739,
viscouscycles.f90:1291-2069)."""
import numpy as np
import pytest


def _deck(ucg, text, driver="ratestate"):
    from unicycle_b200 import Deck
    return Deck(text, driver)


def test_rectangle_config_round_trip(ucg):
    from unicycle_b200 import configs, write_deck
    c = configs.cfg1(nx=8, nz=4)
    pts = [("GPS1", (1000.0, 2000.0, 0.0)), ("GPS2", (-500.0, 300.0, 0.0))]
    d = _deck(ucg, write_deck(c, wdir="out/run1", obs_patches=[1, 17], obs_points=pts, events=[1e8, 2e8]))
    i = d.info
    assert (i["n_rect"], i["n_tri"], i["n_vol"], i["n_obs_state"], i["n_obs_point"], i["n_events"]) == \
        (32, 0, 0, 2, 2, 3)
    assert i["wdir"] == "out/run1" and i["point_names"] == ["GPS1", "GPS2"]
    assert i["mu"] == c["mu"] and i["lambda"] == c["lam"] and i["interval"] == c["t_end"]
    x, L, W, st, dp = c["mesh"]["rect"]
    assert np.array_equal(d.get("rect.x"), np.asarray(x).ravel())
    assert np.array_equal(d.get("rect.length"), L) and np.array_equal(d.get("rect.width"), W)
    np.testing.assert_allclose(d.get("rect.strike"), st, rtol=0, atol=1e-15)
    np.testing.assert_allclose(d.get("rect.dip"), dp, rtol=1e-15)
    fr = c["friction"]
    for q in ("Vpl", "mu0", "sig", "a", "b", "L", "Vo", "damping"):
        assert np.array_equal(d.get("patch." + q), fr[q]), q
    assert np.array_equal(d.get("obs.state"), [1, 17])
    assert np.array_equal(d.get("obs.x"), [1000.0, 2000.0, 0.0, -500.0, 300.0, 0.0])
    assert np.array_equal(d.get("events.time"), [0.0, 1e8, 2e8])
    d.close()


def test_triangle_config_round_trip(ucg):
    from unicycle_b200 import configs, write_deck
    c = configs.cfg2(nx=6, nz=4)
    i1, i2, i3, v = c["mesh"]["tri"]
    d = _deck(ucg, write_deck(c))
    assert d.info["n_tri"] == len(i1) and d.info["n_vertex"] == len(v)
    for name, a in (("tri.i1", i1), ("tri.i2", i2), ("tri.i3", i3)):
        assert np.array_equal(d.get(name), a)
    assert np.array_equal(d.get("tri.vertices"), np.asarray(v).ravel())
    for q in ("Vpl", "a", "b", "L", "sig"):
        assert np.array_equal(d.get("patch." + q), c["friction"][q])


def test_viscous_config_round_trip(ucg):
    from unicycle_b200 import configs, write_deck
    c = configs.cfg3(nxf=4, nzf=2, nxv=2, nyv=2, nzv=2)
    nf = c["n_patch"]
    d = _deck(ucg, write_deck(c, obs_patches=[2], obs_volumes=[1, 3]), driver="viscouscycles")
    i = d.info
    assert (i["n_rect"], i["n_vol"], i["nonlinear_maxwell"], i["thermal"]) == (nf, c["n_vol"], 1, 1)
    x, L, T, W, st = c["mesh"]["vol"]
    assert np.array_equal(d.get("vol.x"), np.asarray(x).ravel())
    assert np.array_equal(d.get("vol.length"), L) and np.array_equal(d.get("vol.thickness"), T)
    assert np.array_equal(d.get("vol.width"), W)
    rh = c["rheology"]
    assert np.array_equal(d.get("vol.e_bg"), np.asarray(rh["ebg"]).ravel())
    assert np.array_equal(d.get("vol.gammadot0m"), rh["gammadot0m"])
    assert np.array_equal(d.get("vol.npowerm"), rh["npowerm"])
    assert np.array_equal(d.get("vol.To"), rh["To"])
    # observation volumes are numbered after all patches, as the reference merges them
    assert np.array_equal(d.get("obs.state"), [2, nf + 1, nf + 3])


LIST_DIRECTED = """\
# a comment
   # an indented comment
 out/dir

# lambda, mu with D exponents and a comma
3.0D4, 3.0d4
1.0E+9
2
1 1d-9 0 0 0 1000 1000 0 90 0
2 1d-9 1000 0 0 1000 1000 0 90 0 / the slash ends the record
2\r
1 0.6 50 0.01 0.014 0.01 1e-6 5.0
2 0.6 50 2*0.01 0.01 1e-6 5.0
0
1
1 2
2
1 'GPS A' 100 200 0
2 P2 300,400,0
3
1.0e8
2.0e8
"""


def test_list_directed_reading(ucg):
    d = _deck(ucg, LIST_DIRECTED)
    i = d.info
    assert i["wdir"] == "out/dir" and i["lambda"] == 3.0e4 and i["mu"] == 3.0e4 and i["interval"] == 1.0e9
    assert np.array_equal(d.get("patch.Vpl"), [1e-9, 1e-9])
    assert np.array_equal(d.get("rect.x"), [0, 0, 0, 1000, 0, 0])
    assert np.array_equal(d.get("patch.a"), [0.01, 0.01]) and np.array_equal(d.get("patch.b"), [0.014, 0.01])
    assert np.array_equal(d.get("rect.dip"), [np.pi / 2, np.pi / 2])
    assert i["point_names"] == ["GPS A", "P2"]
    assert np.array_equal(d.get("obs.x"), [100, 200, 0, 300, 400, 0])
    assert np.array_equal(d.get("events.time"), [0.0, 1e8, 2e8])


def _replace_line(text, k, new):
    lines = text.splitlines()
    lines[k] = new
    return "\n".join(lines) + "\n"


# (line index in LIST_DIRECTED, replacement, expected message fragment, reported line)
BAD = [
    (9, "3 1d-9 1000 0 0 1000 1000 0 90 0", "unexpected index", 10),
    (10, "3", "require frictional properties", 11),
    (5, "3.0D4, -3.0d4", "shear modulus must be positive", 6),
    (6, "0", "simulation time must be positive", 7),
    (8, "1 1d-9 0 0 0 0 0 0 90 0", "length and width must be positive", 9),
    (8, "1 1d-9 0 0 0 1000 1000 0 90", "missing value", 9),
    (8, "1 1d-9 0 0 zero 1000 1000 0 90 0", "not a number", 9),
    (15, "1 3", "observation patch out of range", 16),
    (21, "0.5e8", "timing of perturbations must increase", 22),
]


@pytest.mark.parametrize("k,new,msg,line", BAD)
def test_validation_errors(ucg, k, new, msg, line):
    from unicycle_b200 import UcgError
    with pytest.raises(UcgError) as e:
        _deck(ucg, _replace_line(LIST_DIRECTED, k, new))
    assert msg in str(e.value) and f"line {line}:" in str(e.value), str(e.value)


def test_truncated_and_empty_decks(ucg):
    from unicycle_b200 import UcgError
    with pytest.raises(UcgError, match="unexpected end of input"):
        _deck(ucg, "\n".join(LIST_DIRECTED.splitlines()[:12]))
    with pytest.raises(UcgError, match="nothing to do"):
        _deck(ucg, "out\n1 1\n10\n0\n0\n0\n0\n0\n")


def test_triangle_and_volume_validation(ucg):
    from unicycle_b200 import UcgError
    tri = "out\n3e4 3e4\n10\n0\n1\n1 1e-9 1 2 4 0\n3\n1 0 0 0\n2 1 0 0\n3 0 1 0\n"
    with pytest.raises(UcgError, match="not enough vertices"):
        _deck(ucg, tri)
    vol = ("out\n3e4 3e4\n10\n0\n0\n1\n1 0 0 0 0 0 0 0 0 1000 100 100 100 0 80\n")
    with pytest.raises(UcgError, match="must be vertical"):
        _deck(ucg, vol, "viscouscycles")
    vol2 = ("out\n3e4 3e4\n10\n0\n0\n2\n1 0 0 0 0 0 0 0 0 1000 100 100 100 0 90\n"
            "2 0 0 0 0 0 0 0 0 2000 100 100 100 0 90\n1\n")
    with pytest.raises(UcgError, match="none or all strain volumes"):
        _deck(ucg, vol2, "viscouscycles")
