"""The reference's crossing-angle luminosity anchor (validation/crossing_luminosity_anchor.jl) on the oracle:
symmetric Gaussian beams with negligible charge and no hourglass, each ring a Lorentz boost, the PIC
collision, the reverse boost and the one-turn map; with crabs, the crab-cavity transport of the strong-strong
example around them.  Without crabs the luminosity falls by the Piwinski factor (here against the script's
discrete 15-quantile-slice reference); ideal crabs restore the head-on luminosity.  The line elements and the
PIC collide are the oracle's restatements, which the GPU parity tests pin the device path to."""
import math

import pytest
from scipy.special import erfinv

from oracle import oracle as orc
from octo_b200 import line as ln

THETA = 12.5e-3
SIG = (100e-6, 100e-6, 0.02)
BETA = (0.5, 0.5, 0.02 / 5.0e-4)
CRAB_BETA = (150.0, 30.0, BETA[2])
TUNES = (0.31, 0.32, -0.005)
NS = 15
N = 100_000


def luminosity(angle, crab):
    b1 = orc.beam_gaussian(N, seed=20260728, rng_id=1, beta=BETA, sigma=SIG)
    b2 = orc.beam_gaussian(N, seed=20260728, rng_id=2, beta=BETA, sigma=SIG)
    lb = ln.LorentzBoostSpec(angle)
    if crab:
        strength = (math.tan(angle) / math.sqrt(CRAB_BETA[0] * BETA[0]), 0.0, 0.0)
        t2ip = ln.Linear6DSpec(beta1=CRAB_BETA, beta2=BETA, dmu=(math.pi / 2, 0.0, 0.0))
        tcc = ln.ThinCrabCavitySpec(100e6, N=3, strengthX=strength, strengthY=(0.0,) * 3, phase=(0.0,) * 3)
        before = [t2ip.inverse(), tcc, t2ip, lb]
    else:
        before = [lb]
    elems = [e.to_c() for e in before]
    b1, b2 = orc.track_line(elems, b1), orc.track_line(elems, b2)
    o = orc.Oracle(orc.OracleOptions(grid=(128, 128), nslices1=NS, nslices2=NS, nthreads=8))
    return o.collide(b1, b2, orc.beam_params(-1.0, orc.EMASS_EV, 10e9, 1e8),
                     orc.beam_params(1.0, orc.EMASS_EV, 10e9, 1e8))


def test_crossing_angle_luminosity_anchor():
    l0 = luminosity(0.0, False)
    lx = luminosity(THETA, False)
    lc = luminosity(THETA, True)
    edges = [math.sqrt(2.0) * erfinv(2 * (i / NS) - 1) for i in range(NS + 1)]
    centers = [NS * (math.exp(-edges[i] ** 2 / 2) - math.exp(-edges[i + 1] ** 2 / 2)) / math.sqrt(2 * math.pi)
               * SIG[2] for i in range(NS)]
    r_disc = sum(math.exp(-(math.tan(THETA) * (z1 - z2)) ** 2 / (4 * SIG[0] ** 2))
                 for z1 in centers for z2 in centers) / NS ** 2
    phi = math.tan(THETA) * SIG[2] / SIG[0]
    r_cont = 1 / math.sqrt(1 + phi ** 2)
    assert abs(lx / l0 / r_disc - 1) < 0.02, (lx / l0, r_disc, r_cont)
    assert abs(lc / l0 - 1) < 0.005, lc / l0
