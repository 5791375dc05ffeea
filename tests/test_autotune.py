"""Launch shapes and the autotuner (wcns_get_shape / wcns_set_shape /
wcns_autotune, wcns_b200.autotune).

CPU: the configuration key (stable, and different for anything a shape's
speed depends on) and the JSON cache.
GPU: every shape gives the same steps bit for bit (a shape only moves work
between CTAs); the tuner returns a valid shape, leaves the state alone, and
the cache hands the shape to the next context of the configuration; shapes
the blocks cannot run are refused and the shape in use stays."""
import numpy as np
import pytest

from wcns_b200 import autotune, cases


def _key(**kw):
    base = dict(dims=[(33, 17, 9)], nvis=1, nscheme=41, nflux=3, sa=True, flags=0, precision=64,
                device="B200 sm_100 148 SMs", lib="1:2")
    base.update(kw)
    return autotune.config_key(**base)


def test_config_key_is_stable_and_specific():
    k = _key()
    assert k == _key()
    for change in (dict(dims=[(33, 17, 11)]), dict(nvis=0), dict(nscheme=42), dict(nflux=1), dict(sa=False),
                   dict(flags=2), dict(precision=32), dict(device="other"), dict(lib="1:3")):
        assert _key(**change) != k, change


def test_cache_roundtrip(tmp_path, monkeypatch):
    path = str(tmp_path / "sub" / "shapes.json")
    monkeypatch.setenv("WCNS_SHAPE_CACHE", path)
    assert autotune.cache_path() == path
    assert autotune.load_cache() == {}
    autotune.store("a", {"shape": [4, 1, 16, 8]})
    autotune.store("b", {"shape": [2, 0, 32, 32]})
    d = autotune.load_cache()
    assert d["a"]["shape"] == [4, 1, 16, 8] and d["b"]["shape"] == [2, 0, 32, 32]
    with open(path, "w") as f:
        f.write("not json")
    assert autotune.load_cache() == {}


def _run(case, shape=None, steps=3, tune=False):
    from wcns_b200.solver import Wcns
    g = Wcns(case)
    if case.sa:
        g.sa_setup(case.sa["timedt_turb"], case.sa["kmaxlim"])
    if shape is not None:
        g.set_shape(shape)
    info = autotune.tuned(g, reps=1, use_cache=False) if tune else None
    h = g.step(steps)
    out = [g.get(f, nb) for nb in range(1, case.nblocks + 1) for f in ("r", "u", "v", "w", "p")]
    return g, h, out, info


@pytest.mark.gpu
def test_shapes_do_not_change_results():
    case = cases.small_plate_case()
    g0, h0, s0, _ = _run(case)
    assert g0.shape[0] >= 1  # the small plate sweeps with the clustered kernel
    from wcns_b200.solver import WcnsError
    ran = 0
    for shape in ([1, 0, 4, 8], [2, 0, 16, 4], [4, 1, 8, 32], [8, 0, 32, 16], [16, 0, 4, 4]):
        try:
            g, h, s, _ = _run(case, shape)
        except WcnsError:  # a cluster the largest block's columns do not fit
            continue
        ran += 1
        assert g.shape == shape
        np.testing.assert_array_equal(h, h0)
        for a, b in zip(s, s0):
            np.testing.assert_array_equal(a, b)
        g.close()
    assert ran >= 2


@pytest.mark.gpu
def test_autotune_keeps_state_and_results():
    case = cases.small_channel_case()
    g0, h0, s0, _ = _run(case)
    g, h, s, info = _run(case, tune=True)
    assert info["source"] == "tuned" and len(info["phase_ms"]) == 3
    sh = g.shape
    assert sh == info["shape"] and 4 <= sh[2] <= 32 and 4 <= sh[3] <= 32
    np.testing.assert_array_equal(h, h0)
    for a, b in zip(s, s0):
        np.testing.assert_array_equal(a, b)


@pytest.mark.gpu
def test_cache_hands_shape_to_next_context(tmp_path, monkeypatch):
    from wcns_b200.solver import Wcns
    monkeypatch.setenv("WCNS_SHAPE_CACHE", str(tmp_path / "shapes.json"))
    case = cases.small_plate_case()
    a = Wcns(case)
    ia = autotune.tuned(a, reps=1)
    assert ia["source"] == "tuned"
    b = Wcns(case)
    ib = autotune.tuned(b, reps=1)
    assert ib["source"] == "cache" and b.shape == a.shape


@pytest.mark.gpu
def test_invalid_shapes_are_refused():
    from wcns_b200.solver import Wcns, WcnsError
    g = Wcns(cases.small_plate_case())
    before = g.shape
    for bad in ([-1, 1, 32, 32], [1, 1, 0, 32], [1, 1, 32, 33], [64, 1, 32, 32], [1, 2, 32, 32]):
        with pytest.raises(WcnsError):
            g.set_shape(bad)
        assert g.shape == before


@pytest.mark.gpu
def test_switch_to_wide_sweeps_and_back():
    """shape[0] = 0 sweeps a clustered-capable context with the wide
    cooperative kernels (the same per-point arithmetic: equal to the
    clustered steps within round-off); a cluster shape switches back and
    reproduces the clustered steps bit for bit.  The SA model's scalar sweeps
    follow (the reduced channel with SA)."""
    case = cases.small_plate_case()
    g0, h0, s0, _ = _run(case)
    shape = g0.shape
    g, h, s, _ = _run(case, [0, 0, 32, 32])
    assert g.sweep_mode() == "wide" and g.shape[0] == 0
    np.testing.assert_allclose(h, h0, rtol=1e-12, atol=0)
    for a, b in zip(s, s0):
        assert float(np.max(np.abs(a - b))) <= 1e-12 * max(float(np.max(np.abs(b))), 1.0)
    g.set_shape(shape)
    assert g.sweep_mode() == "clustered"
    from wcns_b200.solver import Wcns
    g2 = Wcns(case)
    g2.set_shape([0, 0, 32, 32])
    g2.set_shape(shape)
    h2 = g2.step(3)
    np.testing.assert_array_equal(h2, h0)
    sa = cases.small_channel_case()
    a, ha, _, _ = _run(sa)
    b, hb, _, _ = _run(sa, [0, 0, 32, 32]) if a.shape[0] else (a, ha, None, None)
    np.testing.assert_allclose(hb, ha, rtol=1e-11, atol=0)
