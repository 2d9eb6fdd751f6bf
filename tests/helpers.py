"""Shared test fixtures: seeded beams (built by the oracle on the host, as Beam() builds them),
and the mapping from a PICPoissonSolver to the oracle's options."""
import numpy as np

from oracle import oracle as orc

E_BEAM = dict(beta=(0.55, 0.056, 0.7e-2 / 5.5e-4), sigma=(106e-6, 9.5e-6, 0.7e-2))
P_BEAM = dict(beta=(0.8, 0.072, 6e-2 / 6.6e-4), sigma=(95e-6, 8.5e-6, 6e-2))
# Contracts.jl:1173-1187
E_PARAMS = dict(charge=-1.0, mass=orc.EMASS_EV, energy=10e9, npart=1.7203e11, r0=orc.RE)
P_PARAMS = dict(charge=1.0, mass=orc.PMASS_EV, energy=275e9, npart=0.6881e11, r0=orc.RE * orc.ME0 / orc.PMASS_EV)


def beams(n1, n2, e_sigma=None, p_sigma=None, seed=123456789):
    eb = dict(E_BEAM)
    pb = dict(P_BEAM)
    if e_sigma is not None:
        eb["sigma"] = e_sigma
    if p_sigma is not None:
        pb["sigma"] = p_sigma
    e = orc.beam_gaussian(n1, seed=seed, rng_id=1, **eb)
    p = orc.beam_gaussian(n2, seed=seed, rng_id=2, **pb)
    return e, p


def oracle_params():
    pe = orc.beam_params(E_PARAMS["charge"], E_PARAMS["mass"], E_PARAMS["energy"], E_PARAMS["npart"], E_PARAMS["r0"])
    pp = orc.beam_params(P_PARAMS["charge"], P_PARAMS["mass"], P_PARAMS["energy"], P_PARAMS["npart"], P_PARAMS["r0"])
    return pe, pp


def oracle_options(solver, nthreads=8, fixed=False):
    s1, s2 = solver.resolved_slicing1, solver.resolved_slicing2
    return orc.OracleOptions(
        grid=solver.grid, deposit_method=solver.deposit_method,
        luminosity_deposit_method=solver.luminosity_deposit_method, luminosity_grid=solver.luminosity_grid,
        green_type=solver.green_type, green_cache=solver.green_cache, field_derivative=solver.field_derivative,
        slice_interpolation=solver.slice_interpolation, interaction_grid=solver.interaction_grid,
        grid_extent=solver.grid_extent, grid_extent_sigma=solver.grid_extent_sigma,
        min_transverse_extent=solver.min_transverse_extent, grid_quantize=solver.grid_quantize,
        slice_pair_green_min_ratio=solver.slice_pair_green_min_ratio,
        slice_pair_green_growth=solver.slice_pair_green_growth, longitudinal_kick=solver.longitudinal_kick,
        nslices1=s1.nslices, nslices2=s2.nslices,
        method1=s1.method, method2=s2.method, resolution1=s1.resolution, resolution2=s2.resolution,
        center_position1=s1.center_position, center_position2=s2.center_position,
        positions1=list(s1.positions), positions2=list(s2.positions),
        kbb1=solver.kbb1, kbb2=solver.kbb2, luminosity_scale=solver.luminosity_scale,
        fixed_point_deposit=fixed, nthreads=nthreads,
        gaussian=hasattr(solver, "margin_sigma"), neutralize=getattr(solver, "neutralize", True),
        margin_sigma=getattr(solver, "margin_sigma", 5.0), coupling_tol=getattr(solver, "coupling_tol", float("inf")))


def within(a, b, atol, rtol):
    """max over elements of |a-b| / (atol + rtol*|b|): <= 1 passes (isapprox per element)."""
    a = np.asarray(a); b = np.asarray(b)
    return float(np.max(np.abs(a - b) / (atol + rtol * np.abs(b))))


def tilt(b, angle):
    """Rotate a beam's transverse plane, (x, y) and (px, py), by `angle` in place: an x-y coupled beam."""
    c, s = np.cos(angle), np.sin(angle)
    x, px, y, py = b[0].copy(), b[1].copy(), b[2].copy(), b[3].copy()
    b[0], b[2] = c * x - s * y, s * x + c * y
    b[1], b[3] = c * px - s * py, s * px + c * py
    return b
