"""Moment observer host logic: moment names, parsing and selection as the reference defines them
(src/tasks/BeamObservers.jl:488-628, docstring examples at :530-551, 680-700), and the oracle's moment row
against a direct numpy evaluation."""
import numpy as np
import pytest

from oracle import oracle as orc
from octo_b200 import observers as ob
from octo_b200.solver import ArgumentError


def test_names_and_parsing():
    assert ob.moment_name(ob.moment(x=1)) == "m100000"
    assert ob.moment_name(ob.moment(x=1, px=1)) == "m110000"
    assert ob.moment_name(ob.moment(pz=4)) == "m000004"
    assert ob.moment_name(ob.moment(x=10)) == "m10_0_0_0_0_0"
    assert ob.moment_name(ob.moment(x=1, px=10)) == "m1_10_0_0_0_0"
    for name in ("m110000", "m1_10_0_0_0_0", "m000004"):
        assert ob.moment_name(ob.parse_moment(name)) == name
    for bad in ("x110000", "m", "m1100", "m1_2_3"):
        with pytest.raises(ArgumentError):
            ob.parse_moment(bad)
    with pytest.raises(ArgumentError):
        ob.moment(-1, 0, 0, 0, 0, 0)


def test_selection():
    default = ob.selected_moments()
    assert len(default) == 27
    assert [ob.moment_name(m) for m in default[:7]] == ["m100000", "m010000", "m001000", "m000100", "m000010",
                                                        "m000001", "m200000"]
    assert ob.moment_name(default[-1]) == "m000002"
    assert len(ob.selected_moments(orders=((1, 2), 3))) == 6 + 21 + 56
    assert ob.selected_moments(orders=()) == ()
    assert ob.selected_moments(orders=(0,)) == ()
    sel = ob.selected_moments(orders=2, extra=["m000004", ob.moment(x=1)], exclude=[ob.moment(x=2)])
    names = [ob.moment_name(m) for m in sel]
    assert names[0] == "m100000" and names[-1] == "m000004" and "m200000" not in names
    # exclude wins over extra
    assert ob.moment(pz=4) not in ob.selected_moments(orders=1, extra="m000004", exclude="m000004")
    # canonical order does not depend on input order
    assert ob.selected_moments(orders=(2, 1)) == default


def test_oracle_moment_row():
    rng = np.random.default_rng(3)
    b = rng.normal(size=(6, 5000)) * np.array([[1e-4], [2e-5], [1e-5], [3e-6], [7e-3], [5e-4]]) + 1e-6
    moments = ob.selected_moments(orders=(1, 2, 3), extra="m000004")
    row = orc.moment_row(b, moments, turn=12)
    assert row[0] == 12.0
    mu = b.mean(axis=1)
    for k, m in enumerate(moments):
        if sum(m) == 1:
            want = mu[m.index(1)]
        else:
            want = np.mean(np.prod([(b[d] - mu[d]) ** m[d] for d in range(6)], axis=0))
        scale = np.prod([b[d].std() ** m[d] for d in range(6)])
        assert abs(row[1 + k] - want) <= 1e-12 * scale
    bad = b.copy()
    bad[2, 10] = np.nan
    # unmasked, the NaN reaches the moments whose powers involve y (a zero power skips its coordinate,
    # BeamObservers.jl:1263-1266)
    np.testing.assert_array_equal(np.isnan(orc.moment_row(bad, moments, 1)[1:]), [m[2] > 0 for m in moments])
    masked = orc.moment_row(bad, moments, 1, mask_lost=True)
    np.testing.assert_allclose(masked, orc.moment_row(np.delete(b, 10, axis=1), moments, 1), rtol=0, atol=0)
    dead = np.full((6, 4), np.inf)
    r = orc.moment_row(dead, moments, 5, mask_lost=True)
    assert r[0] == 5.0 and np.all(np.isnan(r[1:]))
