"""C-ABI and host-side checks that need no GPU: the library loads and exports every declared entry
point, the ctypes structures match the header's layout, the host quantiles match the oracle's, and
the PICPoissonSolver mirror validates like the reference."""
import ctypes as C
import os
import re
import subprocess

import pytest

import octo_b200 as ob
from octo_b200 import _lib
from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "octo_b200.h")


def test_library_loads_and_exports_every_declared_symbol():
    code = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)  # declarations only, not comments
    declared = set(re.findall(r"\b(octo_[a-z0-9_]+)\s*\(", code))
    lib = _lib.lib()
    for name in declared:
        assert hasattr(lib, name), name
    assert declared == set(_lib.EXPORTS)
    assert lib.octo_version() >= 1


def _c_layout():
    src = r"""
#include <stdio.h>
#include <stddef.h>
#include "octo_b200.h"
#define F(T, m) printf(#T " " #m " %zu\n", offsetof(T, m));
int main(void) {
  printf("octo_pic_options size %zu\n", sizeof(octo_pic_options));
  printf("octo_beam size %zu\n", sizeof(octo_beam));
  printf("octo_collide_report size %zu\n", sizeof(octo_collide_report));
  printf("octo_element size %zu\n", sizeof(octo_element));
  F(octo_pic_options, grid_extent_sigma) F(octo_pic_options, longitudinal_kick) F(octo_pic_options, positions1)
  F(octo_pic_options, kbb1) F(octo_pic_options, precision) F(octo_beam, x) F(octo_beam, pz)
  F(octo_pic_options, solver) F(octo_pic_options, include_sigma_xy) F(octo_pic_options, min_sigma)
  F(octo_pic_options, resolution2) F(octo_pic_options, coupling_tol)
  F(octo_collide_report, turn) F(octo_collide_report, kernel_launches) F(octo_collide_report, replayed)
  F(octo_element, rng_id) F(octo_element, p)
  return 0;
}
"""
    import tempfile
    d = tempfile.mkdtemp()
    c = os.path.join(d, "l.c")
    open(c, "w").write(src)
    exe = os.path.join(d, "l")
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    return {tuple(line.split()[:2]): int(line.split()[2]) for line in out.splitlines()}


def test_ctypes_structures_match_header_layout():
    lay = _c_layout()
    assert lay[("octo_pic_options", "size")] == C.sizeof(_lib.OctoPicOptions)
    assert lay[("octo_beam", "size")] == C.sizeof(_lib.OctoBeam)
    assert lay[("octo_collide_report", "size")] == C.sizeof(_lib.OctoCollideReport)
    assert lay[("octo_element", "size")] == C.sizeof(_lib.OctoElement)
    for (t, m), v in lay.items():
        if m == "size":
            continue
        cls = {"octo_pic_options": _lib.OctoPicOptions, "octo_beam": _lib.OctoBeam,
               "octo_collide_report": _lib.OctoCollideReport, "octo_element": _lib.OctoElement}[t]
        assert getattr(cls, m).offset == v, (t, m)


def test_host_quantiles_match_the_oracle_bitwise():
    L = _lib.lib()
    for ns in range(1, 65):
        for s in range(1, ns):
            x = 2 * s / ns - 1
            assert L.octo_erfinv(x) == orc.erfinv(x)
            assert L.octo_normal_quantile(s, ns) == 2 ** 0.5 * orc.erfinv(x)


def test_solver_defaults_and_validation():
    s = ob.PICPoissonSolver()
    assert s.grid == (128, 128) and s.deposit_method == "CIC" and s.green_cache == "slice_pair"
    assert s.slice_pair_green_min_ratio == 0.5 and s.slice_pair_green_growth == 0.25
    with pytest.raises(ob.ArgumentError):
        ob.PICPoissonSolver(field_derivative="sixth")
    with pytest.raises(ob.ArgumentError):
        ob.PICPoissonSolver(grid=(4, 16))
    with pytest.raises(ob.ArgumentError):
        ob.PICPoissonSolver(slice_pair_green_min_ratio=0.0)
    with pytest.raises(ob.ArgumentError):
        ob.PICPoissonSolver(interaction_grid="node", slice_interpolation="quadratic")
    with pytest.raises(ob.ArgumentError):
        ob.PICPoissonSolver(interaction_grid="node", grid_extent="sigma")
    with pytest.raises(ob.ArgumentError):
        ob.LongitudinalSlicing(nslices=3, method="specified", positions=[0.0])


def test_gpu_backend_rejects_what_it_does_not_implement():
    sl = ob.LongitudinalSlicing(nslices=3, method="normal_quantile")
    for kw in (dict(green_type="lattice"), dict(grid=(80, 80)), dict(grid=(96, 36)), dict(grid=(1024, 64))):
        with pytest.raises(ob.ArgumentError):
            ob.PICPoissonSolver(slicing=sl, **kw).to_c()
    for ig, code in (("slice_pair", 0), ("source_slice", 1), ("node", 2)):
        assert ob.PICPoissonSolver(slicing=sl, interaction_grid=ig).to_c().interaction_grid == code
    with pytest.raises(ob.ArgumentError):  # union-sized meshes apply no extent estimator
        ob.PICPoissonSolver(slicing=sl, interaction_grid="source_slice", grid_extent="sigma")
    o = ob.PICPoissonSolver(slicing=sl, grid_extent="sigma", grid_extent_sigma=4.5).to_c()  # :slice_pair only
    assert (o.grid_extent, o.grid_extent_sigma) == (1, 4.5)
    with pytest.raises(ob.ArgumentError):  # the :equal_area histogram's shared-memory bound
        ob.PICPoissonSolver(slicing=ob.LongitudinalSlicing(nslices=64, method="equal_area", resolution=300)).to_c()
    for m, code in (("equal_area", 2), ("equal_count", 3), ("equal_width", 4), ("equal_spaced", 4), ("gaussian", 0)):
        o = ob.PICPoissonSolver(slicing=ob.LongitudinalSlicing(nslices=3, method=m, resolution=7)).to_c()
        assert (o.slicing_method1, o.slicing_method2, o.resolution1) == (code, code, 7)
    for g in ((48, 48), (96, 64), (384, 192), (512, 512)):  # 2^a and 3*2^a FFT lines
        assert ob.PICPoissonSolver(slicing=sl, grid=g).to_c().nx == g[0]
    o = ob.PICPoissonSolver(slicing=sl, deposit_method="TSC", field_derivative="fourth").to_c()
    assert (o.nx, o.deposit_method, o.field_derivative, o.nslices1) == (128, 1, 4, 3)


def test_soft_gaussian_solver_options():
    """GaussianPoissonSolver's keyword validation (interface.jl:976-1000) and its C options."""
    import math
    import octo_b200 as ob
    for kw in (dict(min_sigma=-1.0), dict(min_sigma=math.inf), dict(gaussian_when_luminosity=3),
               dict(batch_mode="parallel"), dict(virtual_drift="paraxial")):
        with pytest.raises(ob.ArgumentError):
            ob.GaussianPoissonSolver(**kw)
    s = ob.GaussianPoissonSolver(slicing1=ob.LongitudinalSlicing(nslices=3, method="normal_quantile"),
                                 slicing2=ob.LongitudinalSlicing(nslices=5, method="normal_quantile"),
                                 min_sigma=2e-6, gaussian_when_luminosity=1, ignore_centroid2=True,
                                 virtual_drift="exact", include_sigma_xy=True, kbb1=1e-4)
    o = s.to_c()
    assert (o.solver, o.nslices1, o.nslices2, o.gaussian_when_luminosity) == (_lib.SOLVER_SOFT_GAUSSIAN, 3, 5, 1)
    assert (o.ignore_centroid1, o.ignore_centroid2, o.virtual_drift, o.include_sigma_xy) == (0, 1, 2, 1)
    assert o.min_sigma == 2e-6 and o.has_kbb1 == 1 and o.kbb1 == 1e-4 and o.has_kbb2 == 0
