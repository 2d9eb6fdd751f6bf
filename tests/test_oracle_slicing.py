"""The oracle's restatement of the reference's other slicing methods (slicing.jl:104-156 :equal_area,
330-365 :equal_count, 367-388 :equal_width), pinned on the reference's own slicing tests
(runtests.jl:4540-4590): the zero-width convention (every particle in slice 1 for :equal_area and
:equal_width), :equal_count membership by rank (no boundary violations for continuous z; under ties a
violating particle sits exactly on its boundary), and the properties each method promises (exact equal
counts, nearly equal areas, equal widths with exact endpoints)."""
import numpy as np
import pytest

from oracle import oracle as orc


def _members(order, cnt):
    out, k = [], 0
    for c in cnt:
        out.append(order[k:k + c])
        k += c
    return out


@pytest.mark.parametrize("method", ["equal_area", "equal_width", "normal_quantile"])
def test_zero_width_beam_lands_in_slice_one(method):
    z = np.full(8, 1.5e-3)
    b, c, w, cnt, order = orc.slices(z, 4, method=method)
    assert list(cnt) == [8, 0, 0, 0]


def test_equal_count_membership_is_by_rank():
    i = np.arange(1, 2001)
    zc = 2.0e-2 * np.sin(0.7 * i + 2.0)
    zq = np.round(2.0e-2 * np.sin(0.7 * i + 2.0), 3)

    def violations(z):
        b, c, w, cnt, order = orc.slices(z, 9, method="equal_count")
        bad = []
        for k, idx in enumerate(_members(order, cnt)):
            lb, rb = b[k], b[k + 1]
            for p in idx:
                inside = (lb <= z[p] <= rb) if k == 8 else (lb <= z[p] < rb)
                if not inside:
                    bad.append((k, p))
        return b, cnt, bad

    _, cnt, bad = violations(zc)
    edges = [int(np.floor(s * 2000 / 9)) for s in range(10)]  # first_pos / last_pos of slicing.jl:345-350
    assert not bad and list(cnt) == list(np.diff(edges))
    bq, _, badq = violations(zq)
    assert badq and all(zq[p] == bq[k + 1] for k, p in badq)


def test_equal_count_ranks_ties_by_index():
    z = np.array([3.0, 1.0, 1.0, 2.0, 1.0, -0.0, 0.0])
    b, c, w, cnt, order = orc.slices(z, 3, method="equal_count")
    assert list(order) == [5, 6, 1, 2, 4, 3, 0]  # sortperm: -0.0 before 0.0, equal values by index
    assert list(cnt) == [2, 2, 3]


def test_equal_area_counts_are_nearly_equal():
    z = np.random.default_rng(3).standard_normal(100_000) * 7e-3
    b, c, w, cnt, order = orc.slices(z, 15, method="equal_area")
    assert b[0] == z.min() and b[-1] == z.max() and np.all(np.diff(b) > 0)
    assert np.max(np.abs(cnt - 100_000 / 15)) < 0.02 * 100_000 / 15


def test_equal_width_boundaries():
    z = np.random.default_rng(4).standard_normal(50_000) * 7e-3
    b, c, w, cnt, order = orc.slices(z, 7, method="equal_width")
    assert b[0] == z.min() and b[-1] == z.max()
    exact = z.min() + (z.max() - z.min()) * np.arange(8) / 7
    assert np.all(np.abs(b - exact) <= 2 * np.spacing(np.abs(exact).max()))
    for lo, hi in ((-1.0, 1.0), (0.0, 1.0), (-0.0213, 0.0347), (1e-3, 7.5e-3)):
        r = orc.julia_range(lo, hi, 11)
        assert r[0] == lo and r[-1] == hi and np.all(np.diff(r) > 0)
        assert np.all(np.abs(r - np.linspace(lo, hi, 11)) <= np.spacing(max(abs(lo), abs(hi))))
    assert list(orc.julia_range(0.0, 1.0, 11)) == [k / 10 for k in range(11)]
