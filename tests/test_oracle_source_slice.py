"""The oracle's interaction_grid = :source_slice (pic_cpu.jl:30-60, 360-380, 602-712): one mesh per (source
slice, direction), sized from a union box taken at the source slice's first use, pairs run one at a time in
collision order.  The properties are the reference's own (runtests.jl:5174-5200, 9800-9845, 7755): same physics
as :slice_pair to 1e-3 in luminosity, a different kick, every partner particle inside the shared box, the
sequential schedule whatever the thread count, and a non-finite partner coordinate named at the union bounds."""
import numpy as np
import pytest

from helpers import beams, oracle_params
from oracle import oracle as orc


def _opts(**kw):
    base = dict(grid=(64, 64), nslices1=4, nslices2=4, nthreads=8)
    base.update(kw)
    return orc.OracleOptions(**base)


def _collide(opt, e, p):
    e, p = e.copy(), p.copy()
    o = orc.Oracle(opt)
    pe, pp = oracle_params()
    lum = o.collide(e, p, pe, pp)
    return e, p, lum, o


def test_source_slice_same_physics_different_kick():
    e, p = beams(6000, 6000)
    e_sp, p_sp, l_sp, _ = _collide(_opts(), e, p)
    e_ss, p_ss, l_ss, o = _collide(_opts(interaction_grid="source_slice"), e, p)
    assert not np.array_equal(e_sp, e_ss)
    assert np.all(np.isfinite(e_ss)) and np.all(np.isfinite(p_ss))
    assert abs(l_ss / l_sp - 1) < 1e-3
    # the kicks themselves agree to the mesh resolution: a few per cent of the kick's spread
    for row in (1, 3):
        dk_sp, dk_ss = e_sp[row] - e[row], e_ss[row] - e[row]
        assert np.sqrt(np.mean((dk_ss - dk_sp) ** 2)) < 0.05 * np.std(dk_sp)
    assert o.dropped() == 0


def test_source_slice_is_sequential_whatever_the_thread_count():
    e, p = beams(3000, 3000)
    a = _collide(_opts(interaction_grid="source_slice", nthreads=1, nslices1=5, nslices2=3), e, p)
    b = _collide(_opts(interaction_grid="source_slice", nthreads=8, nslices1=5, nslices2=3), e, p)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]


def test_source_slice_shares_one_mesh_per_source_slice():
    """green_cache = :none: each pair sizes its mesh from the shared union box, so every pair of source slice 2
    (direction 1) deposits on the same mesh; under :slice_pair the meshes follow each partner slice."""
    e, p = beams(4000, 4000)
    meshes = {}
    for mode in ("source_slice", "slice_pair"):
        got = []
        for j in range(1, 5):
            o = orc.Oracle(_opts(interaction_grid=mode, green_cache="none", fixed_point_deposit=True))
            o.capture_plane(2, j, 1, 0)
            pe, pp = oracle_params()
            o.collide(e.copy(), p.copy(), pe, pp)
            got.append(o.captured_plane()[1])
        meshes[mode] = got
    assert all(m == meshes["source_slice"][0] for m in meshes["source_slice"])
    assert len(set(meshes["slice_pair"])) > 1
    # the shared mesh is the union: wider than any one pair's
    w_ss = meshes["source_slice"][0][2]
    assert all(w_ss >= m[2] for m in meshes["slice_pair"])


def test_source_slice_union_box_holds_every_partner_particle():
    """runtests.jl:9829-9843: the field half of the union box covers every partner particle at its own collision
    point, and the source half every source particle at every drift across the partner's z range (its two
    extremes bound the affine drift)."""
    e, p = beams(5000, 5000)
    _, c, _, _, _ = orc.slices(e[4], 4)
    ids = np.argsort(e[4])[1250:2500]          # a slice's worth of the electron beam
    src = e[:, ids]
    centre = float(c[1])
    (sx0, sx1, sy0, sy1), (fx0, fx1, fy0, fy1) = orc.union_bounds(src[:4], centre, p[:5])
    s = 0.5 * (p[4] - centre)
    fx, fy = p[0] + s * p[1], p[2] + s * p[3]
    assert fx.min() == fx0 and fx.max() == fx1 and fy.min() == fy0 and fy.max() == fy1
    for drift in np.linspace(0.5 * (centre - p[4].max()), 0.5 * (centre - p[4].min()), 7):
        x, y = src[0] + src[1] * drift, src[2] + src[3] * drift
        assert sx0 <= x.min() and x.max() <= sx1 and sy0 <= y.min() and y.max() <= sy1
    assert orc.union_bounds(src[:4], centre, p[:5, :0]) is None
    bad = p[:5].copy()
    bad[4, 7] = np.nan
    with pytest.raises(orc.OracleErrorPy) as err:
        orc.union_bounds(src[:4], centre, bad)
    assert err.value.code == orc.ERR_NONFINITE


def test_source_slice_drops_are_counted():
    """The box is taken at the source slice's first use and the partner's particles are kicked afterwards, so a
    particle can leave it (pic_cpu.jl:1082-1096); such a particle is counted, never silently dropped.  With no
    cache growth a few do leave on this pair; with the default growth none."""
    e, p = beams(5000, 5000)
    _, _, _, tight = _collide(_opts(interaction_grid="source_slice", slice_pair_green_growth=0.0), e, p)
    _, _, _, grown = _collide(_opts(interaction_grid="source_slice"), e, p)
    assert 0 < tight.dropped() < 10 and grown.dropped() == 0


def test_source_slice_cache_holds_one_entry_per_source_slice():
    e, p = beams(4000, 4000)
    _, _, _, o = _collide(_opts(interaction_grid="source_slice", nslices1=5, nslices2=3), e, p)
    hits, misses, rebuilds = o.cache_stats()
    assert misses == 5 + 3
    assert hits + misses + rebuilds == 2 * 5 * 3


def test_source_slice_quadratic_runs():
    e, p = beams(3000, 3000)
    e_l, _, l_l, _ = _collide(_opts(interaction_grid="source_slice"), e, p)
    e_q, _, l_q, _ = _collide(_opts(interaction_grid="source_slice", slice_interpolation="quadratic"), e, p)
    assert not np.array_equal(e_l, e_q) and abs(l_q / l_l - 1) < 1e-3


def test_source_slice_rejects_sigma_extent():
    e, p = beams(500, 500)
    with pytest.raises(orc.OracleErrorPy) as err:
        _collide(_opts(interaction_grid="source_slice", grid_extent="sigma"), e, p)
    assert err.value.code == orc.ERR_UNSUPPORTED


def test_source_slice_nonfinite_partner_fails_at_the_union_bounds():
    e, p = beams(800, 800)
    p[2, 123] = np.nan
    with pytest.raises(orc.OracleErrorPy) as err:
        _collide(_opts(interaction_grid="source_slice"), e, p)
    assert err.value.code == orc.ERR_NONFINITE and "union bounds" in str(err.value)
