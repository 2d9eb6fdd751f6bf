"""Line elements on the host: the oracle's restatement against the reference's own element tests
(test/runtests.jl:188-206, 207-240, 341-364, 366-436, 450-508, 7434-7442), the spec constructors'
validation, the counter-RNG draws of both methods, and the physics the elements promise (symplectic
maps, the boost pair's Jacobian determinants sec^3 / cos^3, diffusion variance)."""
import math

import numpy as np
import pytest

from oracle import oracle as orc
from octo_b200 import line as ln
from octo_b200.solver import ArgumentError

COORDS0 = (1.0e-3, -2.0e-4, 0.7e-3, 1.0e-4, -2.0e-3, 3.0e-4)


def one(coords):
    return np.array(coords, dtype=np.float64).reshape(6, 1)


def track(elems, beam, **kw):
    return orc.track_line([e.to_c() if hasattr(e, "to_c") else e for e in elems], beam, **kw)


def radiation_spec(**kw):
    """The spec of runtests.jl:367-379."""
    base = dict(damping_turns=(10.0, 20.0, 30.0), beta=(0.7, 0.9, 1.1), alpha=(0.2, -0.1, 0.05),
                sigma=(1.2e-3, 0.8e-3, 2.0e-3), zeta=(0.01, -0.02, 0.03, -0.04), eta=(0.05, -0.06, 0.07, -0.08),
                R=(0.01, 0.02, -0.015, 0.005), rng_id=0x4567)
    base.update(kw)
    return ln.LumpedRadSpec(**base)


def ramp_beam(n=128):
    """The Phase6DRep of runtests.jl:351-358."""
    return np.stack([np.linspace(-1.0e-3, 1.0e-3, n), np.linspace(2.0e-4, -2.0e-4, n), np.linspace(0.7e-3, -0.7e-3, n),
                     np.linspace(-1.0e-4, 1.0e-4, n), np.linspace(-2.0e-3, 2.0e-3, n), np.linspace(3.0e-4, -3.0e-4, n)])


def test_radiation_method_and_flag_semantics():
    # runtests.jl:381-408: Damping6DMap == radiation without excitation, Diffusion6DMap == radiation
    # without damping; a disabled component leaves the particle untouched
    b = one(COORDS0)
    kw = dict(turn=17, seed=0x12345678, rng_method=1)
    both = radiation_spec(is_damping=True, is_excitation=True)
    damping = track([both.to_c("damping")], b, **kw)
    diffusion = track([both.to_c("diffusion")], b, **kw)
    assert np.array_equal(damping, track([radiation_spec(is_excitation=False)], b, **kw))
    assert np.array_equal(diffusion, track([radiation_spec(is_damping=False)], b, **kw))
    rt = both.compile_runtime("damping")
    assert rt.is_damping and not rt.is_excitation
    rt = both.compile_runtime("diffusion")
    assert not rt.is_damping and rt.is_excitation
    assert np.array_equal(track([radiation_spec(is_damping=False).to_c("damping")], b, **kw), b)
    assert np.array_equal(track([radiation_spec(is_excitation=False).to_c("diffusion")], b, **kw), b)
    assert not np.array_equal(damping, b) and not np.array_equal(diffusion, b)


def test_radiation_constants_and_validation():
    # runtests.jl:410-436
    long_turn = ln.LumpedRadSpec(damping_turns=(1e8, 1e8, 1e8), beta=(1, 1, 1), sigma=(1, 1, 1), rng_id=1)
    rt = long_turn.compile_runtime()
    assert rt.excitation[0] == math.sqrt(-math.expm1(-2.0 / 1e8)) and rt.excitation[0] > 0
    inf_turn = ln.LumpedRadSpec(damping_turns=(math.inf,) * 3, sigma=(1.0, 1.0, 1.0), rng_id=1).compile_runtime()
    assert inf_turn.damping == (1.0, 1.0, 1.0) and inf_turn.excitation == (0.0,) * 9
    for kw in (dict(damping_turns=(10.0, 0.0, 30.0)), dict(damping_turns=(10.0, math.nan, 30.0)),
               dict(damping_turns=(10.0, 20.0, 30.0), beta=(1.0, 0.0, 1.0)),
               dict(damping_turns=(10.0, 20.0, 30.0), sigma=(1.0, -1.0, 1.0)),
               dict(damping_turns=(10.0, 20.0, 30.0), sigma=(1.0, math.inf, 1.0))):
        with pytest.raises(ArgumentError):
            ln.LumpedRadSpec(**kw).compile_runtime()
    with pytest.raises(ArgumentError):
        ln.LumpedRadSpec(damping_turns=(1.0, 1.0, 1.0), tracking_method="symplectic")
    # sigma all negative disables excitation (radiation.jl:153-159)
    assert not ln.LumpedRadSpec(damping_turns=(5.0, 5.0, 5.0), rng_id=2).compile_runtime().is_excitation


def test_rng_ids_are_claimed_and_assigned():
    # counter_rng.jl:50-81: explicit ids are claimed so automatic ones never reissue them
    ln.reset_rng_id_counter(0)
    a = ln.LumpedRadSpec(damping_turns=(5.0, 5.0, 5.0))
    assert a.rng_id == 1
    ln.LumpedRadSpec(damping_turns=(5.0, 5.0, 5.0), rng_id=40)
    assert ln.LumpedRadSpec(damping_turns=(5.0, 5.0, 5.0)).rng_id == 41


def test_chunked_radiation_equals_continuous():
    # runtests.jl:341-364: 7 turns in one call == 3 + 4 turns
    spec = ln.LumpedRadSpec(damping_turns=(20.0, 25.0, 30.0), beta=(0.7, 0.9, 1.1), alpha=(0.2, -0.1, 0.05),
                            sigma=(1.2e-3, 0.8e-3, 2.0e-3), rng_id=0x1234)
    b = ramp_beam()
    for method in (1, 2):
        cont = track([spec], b, turn=0, turns=7, seed=0x5EED, rng_method=method)
        part = track([spec], b, turn=0, turns=3, seed=0x5EED, rng_method=method)
        part = track([spec], part, turn=3, turns=4, seed=0x5EED, rng_method=method)
        assert np.array_equal(cont, part)


def _splitmix64(x):
    m = 0xFFFFFFFFFFFFFFFF
    z = (x + 0x9E3779B97F4A7C15) & m
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    return z ^ (z >> 31)


def _uniform(v):
    return ((v >> 12) + 0.5) * 2.220446049250313e-16


def test_octopus_normal_both_methods():
    # counter_rng.jl:103-176 restated in Python: SplitMix hash of the five counters, Philox4x32-10 keyed by
    # SplitMix mixes of (seed, rng_id, component); Box-Muller pairs, odd component -> cos branch
    m64 = 0xFFFFFFFFFFFFFFFF

    def splitmix_u64(seed, turn, rid, part, comp):
        x = seed
        x ^= _splitmix64((turn + 0x9E3779B97F4A7C15) & m64)
        x ^= _splitmix64((rid + 0xBF58476D1CE4E5B9) & m64)
        x ^= _splitmix64((part + 0x94D049BB133111EB) & m64)
        x ^= _splitmix64((comp + 0xD2B74407B1CE6E93) & m64)
        return _splitmix64(x)

    def philox_u64(seed, turn, rid, part, comp):
        key = _splitmix64(seed) ^ _splitmix64((rid + 0x9E3779B97F4A7C15) & m64) ^ \
            _splitmix64((comp + 0xBF58476D1CE4E5B9) & m64)
        out = orc.philox4x32_block([part & 0xFFFFFFFF, part >> 32, turn & 0xFFFFFFFF, turn >> 32],
                                   [key & 0xFFFFFFFF, key >> 32])
        return (int(out[0]) << 32) | int(out[1])

    for method, u64 in ((1, philox_u64), (2, splitmix_u64)):
        for seed, turn, rid, part in ((0, 0, 1, 1), (0x5EED, 17, 0x4567, 11), (2**63 + 5, 2**33, 3, 2**40)):
            for comp in range(1, 7):
                pair = (comp + 1) // 2
                u1, u2 = _uniform(u64(seed, turn, rid, part, 2 * pair - 1)), _uniform(u64(seed, turn, rid, part, 2 * pair))
                r = math.sqrt(-2.0 * math.log(u1))
                want = r * (math.cos if comp % 2 else math.sin)(6.283185307179586476925286766559 * u2)
                got = orc.octopus_normal(seed, method, turn, rid, part, comp)
                assert abs(got - want) <= 4e-16 * max(1.0, abs(want))


def test_diffusion_variance():
    # runtests.jl:487-500: pure diffusion variance grows as turns * exc^2
    spec = ln.LumpedRadSpec(damping_turns=(1e18,) * 3, beta=(1.0, 1.0, 1.0), sigma=(1.0e-3,) * 3,
                            tracking_method="diffusion", rng_id=0x77)
    b = np.zeros((6, 200_000))
    out = track([spec], b, turn=0, turns=16, seed=777, rng_method=1)
    exc = spec.compile_runtime().excitation[0]
    ratio = np.var(out[0], ddof=1) / (16 * exc ** 2)
    assert 0.95 < ratio < 1.05


def test_linear6d_symplectic_validation():
    # runtests.jl:207-240
    ident = np.eye(6)
    ln.Linear6DSpec(matrix=ident)
    scaled = np.eye(6)
    scaled[0, 0], scaled[1, 1] = 1e8, 1e-8
    ln.Linear6DSpec(matrix=scaled)
    shear = np.eye(6)
    shear[0, 1] = 0.3
    assert ln.Linear6DSpec(matrix=shear).matrix == list(shear.reshape(-1))
    bad = np.eye(6)
    bad[0, 2] = 0.3
    assert np.linalg.det(bad) == 1.0
    with pytest.raises(ArgumentError):
        ln.Linear6DSpec(matrix=bad)
    nonfinite = np.eye(6)
    nonfinite[0, 0] = math.inf
    with pytest.raises(ArgumentError):
        ln.Linear6DSpec(matrix=nonfinite)
    with pytest.raises(ArgumentError):
        ln.Linear6DSpec(beta1=(1.0, 1.0, 1.0))


def test_linear6d_optics_matrix():
    # equal-Twiss optics form is the one-turn rotation the oracle builds (linear6d.jl:233-275)
    beta, alpha, tune = (0.55, 0.056, 12.7), (0.1, -0.2, 0.0), (0.08, 0.14, -0.069)
    spec = ln.Linear6DSpec(beta1=beta, alpha1=alpha, dmu=tuple(2 * math.pi * t for t in tune))
    np.testing.assert_allclose(spec.matrix, orc.linear6d_matrix(beta, alpha, tune), rtol=0, atol=1e-15)
    # dispersion and coupling compose into a symplectic matrix, and zeta2 = zeta1 etc. by default
    full = ln.Linear6DSpec(beta1=beta, beta2=(0.6, 0.05, 12.7), alpha1=alpha, dmu=(1.0, 2.0, 0.1),
                           zeta1=(0.01, -0.02, 0.0, 0.03), eta1=(0.1, 0.02, -0.01, 0.0), R1=(0.02, 0.01, -0.01, 0.03))
    assert ln.linear6d_symplectic_ratio(full.matrix) <= 1.0
    inv = full.inverse()
    prod = np.array(inv.matrix).reshape(6, 6) @ np.array(full.matrix).reshape(6, 6)
    np.testing.assert_allclose(prod, np.eye(6), atol=1e-12)


def test_crab_cavity_validation():
    # runtests.jl:7439-7441, crab_cavity.jl:117-121, 149-155
    for f in (0.0, math.inf, math.nan):
        with pytest.raises(ArgumentError):
            ln.ThinCrabCavitySpec(f, N=1)
    with pytest.raises(ArgumentError):
        ln.ThinCrabCavitySpec(1e8, N=2, strengthX=(1.0,))
    c = ln.ThinCrabCavitySpec(1e8, N=2, strengthX=(1.0, 0.5))
    assert c.strengthY == (0.0, 0.0) and c.phase == (0.0, 0.0)
    with pytest.raises(ArgumentError):
        ln.XYCouplingSpec(r1=1.0, r4=-1.0, r2=0.0, r3=0.0)  # 1 + r1 r4 - r2 r3 = 0


def _jacobian(elem, x0, h=1e-7):
    x0 = np.asarray(x0, dtype=np.float64)
    J = np.zeros((6, 6))
    for k in range(6):
        d = np.zeros(6)
        d[k] = h * max(abs(x0[k]), 1e-3)
        plus = track([elem], one(x0 + d))[:, 0]
        minus = track([elem], one(x0 - d))[:, 0]
        J[:, k] = (plus - minus) / (2 * d[k])
    return J


S6 = np.kron(np.eye(3), np.array([[0.0, 1.0], [-1.0, 0.0]]))


@pytest.mark.parametrize("elem", [
    ln.ThinCrabCavitySpec(197e6, N=3, strengthX=(0.01, -0.003, 0.001), strengthY=(0.002, 0.0, 0.001),
                          phase=(0.1, 0.0, -0.2)),
    ln.ChromaticityKickSpec(xi=(2.0, 1.5), beta=(0.8, 0.07), alpha=(0.3, -0.2), zeta=(0.01, -0.02, 0.03, -0.04),
                            eta=(0.05, -0.06, 0.07, -0.08), R=(0.01, 0.02, -0.015, 0.005)),
    ln.XYCouplingSpec(0.01, 0.02, -0.015, 0.005, mode="B"),
    ln.CrabDispersionSpec(0.01, -0.02, 0.03, -0.04),
    ln.MomentumDispersionSpec(0.05, -0.06, 0.07, -0.08),
])
def test_symplectic_elements(elem):
    J = _jacobian(elem, COORDS0)
    np.testing.assert_allclose(J.T @ S6 @ J, S6, atol=2e-6)


def test_boost_pair_jacobians():
    # lorentz_boost.jl:43-51, 82-88: det = sec(angle)^3 forward, cos(angle)^3 reverse
    a = 0.0125
    Jf = _jacobian(ln.LorentzBoostSpec(a), COORDS0)
    Jr = _jacobian(ln.RevLorentzBoostSpec(a), COORDS0)
    assert abs(np.linalg.det(Jf) * math.cos(a) ** 3 - 1.0) < 1e-6
    assert abs(np.linalg.det(Jr) / math.cos(a) ** 3 - 1.0) < 1e-6
    b = ramp_beam()
    rt = track([ln.LorentzBoostSpec(a), ln.RevLorentzBoostSpec(a)], b)
    np.testing.assert_allclose(rt, b, rtol=0, atol=1e-17)


def test_example_lines_compile():
    for beam in ("electron", "proton"):
        before, after = ln.eic_like_segments(beam)
        arr, n = ln.compile_line((before, after))
        assert n == len(before) + len(after) and n <= 11
        kinds = [arr[k].kind for k in range(n)]
        assert kinds[3] == 3 and kinds[4] == 4  # the boost pair frames the collision
    with pytest.raises(ArgumentError):
        ln.compile_line([object()])


def test_linear6d_full_optics_case_is_symplectic():
    """runtests.jl:250-268: optics with different ends and every dispersion / coupling tuple compiles, i.e.
    its composed matrix passes the symplectic check."""
    spec = ln.Linear6DSpec(beta1=(0.55, 0.056, 12.7), beta2=(0.8, 0.072, 90.9), alpha1=(0.08, 0.14, -0.069),
                           alpha2=(0.0, 0.0, 0.0), dmu=(0.3, 0.4, 0.2), zeta1=(0.01, -0.02, 0.03, -0.01),
                           eta1=(0.02, 0.01, -0.01, 0.04), R1=(0.01, -0.02, 0.015, 0.005),
                           zeta2=(-0.01, 0.01, 0.02, 0.03), eta2=(0.01, -0.03, 0.02, -0.01),
                           R2=(-0.005, 0.01, -0.015, 0.02))
    assert ln.linear6d_symplectic_ratio(spec.matrix) <= 1.0
    S6 = np.kron(np.eye(3), np.array([[0.0, 1.0], [-1.0, 0.0]]))
    M = np.array(spec.matrix).reshape(6, 6)
    np.testing.assert_allclose(M.T @ S6 @ M, S6, atol=1e-13)
