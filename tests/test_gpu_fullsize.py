"""Parity at the full sizes of the benchmark configurations.

The CUDA path (through the C ABI) against the CPU oracle (threaded over the
host's cores; the threads split the elements, so the oracle's arithmetic is
the same as on one thread):

* 2D isentropic vortex, periodic [-10,10]^2, 128 x 128 perturbed quads, P = 4,
  Roe, RK4, CFL 0.5 (1,638,400 DOF), 10 steps;
* 2D Euler channel over a Gaussian bump, 96 x 32 quadratic quads clustered to
  the wall, P = 3, Roe inside, characteristic inlet / outlet at Mach 0.5,
  slip walls, RK4, CFL 0.5, 20 steps;
* 3D Navier-Stokes Taylor-Green vortex, periodic [0,2pi]^3, 32^3 hexes, P = 3,
  Re 1600, Ma 0.1, Rusanov + LDG, RK4 (10,485,760 DOF), 2 steps.

FP64 mode: the state after the steps (and the CFL dt of every step) within
1e-12 relative (max norm) of the FP64 oracle.  Mixed mode: within 1e-6
relative L2 of the FP64 oracle, the mixed-precision bound the path states.
"""
import os

import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_L2_TOL = 1e-6

TGV_MA = 0.1


def _configs():
    from fr_learn_b200 import box2d, box3d, bump2d

    c = np.sqrt(1.4)
    return {
        "vortex_128x128_p4": (lambda: box2d(128, 128, -10.0, 10.0, -10.0, 10.0, perturb=0.1, seed=0), 1, 0.0,
                              dict(order=4, riemannType=1, timeType=4, dtType=1, CFL=0.5, rhoBound=1.0,
                                   uBound=1.0, vBound=1.0, pBound=1.0), 10),
        "bump_96x32_p3": (lambda: bump2d(96, 32, bc_top="symmetry"), 0, 0.0,
                          dict(order=3, riemannType=1, timeType=4, dtType=1, CFL=0.5, rhoBound=1.0,
                               uBound=0.5 * c, pBound=1.0), 20),
        "tgv_32x32x32_p3": (lambda: box3d(32, 32, 32, (0.0, 0.0, 0.0), (2 * np.pi,) * 3), 10, TGV_MA,
                            dict(order=3, viscous=1, riemannType=0, timeType=4, dtType=0, dt=5e-4,
                                 mu_inf=1.0 / 1600.0, prandtl=0.71, fixVis=1, penFact=0.0, tau=1.0), 2),
    }


_ORACLE_CACHE = {}


def _oracle_run(oracle, name):
    """Final state, per-step dt and time of the FP64 oracle (cached: the
    FP64 and mixed tests compare against the same run)."""
    if name not in _ORACLE_CACHE:
        make, ic, a0, kw, nsteps = _configs()[name]
        mesh = make()
        oracle.lib().orc_set_threads(os.cpu_count() or 1)
        o = oracle.Oracle(oracle.params(nDims=mesh.nDims, **kw), mesh)
        o.set_ic(ic, a0)
        dts = []
        for _ in range(nsteps):
            o.update(1)
            dts.append(o.dt)
        _ORACLE_CACHE[name] = (mesh, o.U().copy(), np.array(dts), o.time)
        o.close()
    return _ORACLE_CACHE[name]


@pytest.mark.parametrize("name", list(_configs()))
def test_fullsize_fp64_matches_oracle(oracle, name):
    from fr_learn_b200 import FRG_FP64, Solver

    _, ic, a0, kw, nsteps = _configs()[name]
    mesh, R, dts, t = _oracle_run(oracle, name)
    g = Solver(mesh, precision=FRG_FP64, **kw)
    g.setInitialCondition(ic, a0)
    gdt = []
    for _ in range(nsteps):
        g.update(1)
        gdt.append(g.dt)
    assert relerr(gdt, dts) < FP64_TOL
    assert relerr(g.get("U_spts"), R) < FP64_TOL
    assert abs(g.time - t) <= 1e-12 * t


@pytest.mark.parametrize("name", list(_configs()))
def test_fullsize_mixed_within_bound_of_fp64_oracle(oracle, name):
    from fr_learn_b200 import FRG_MIXED, Solver

    _, ic, a0, kw, nsteps = _configs()[name]
    mesh, R, dts, t = _oracle_run(oracle, name)
    g = Solver(mesh, precision=FRG_MIXED, **kw)
    g.setInitialCondition(ic, a0)
    g.update(nsteps)
    U = g.get("U_spts")
    l2 = float(np.linalg.norm(U - R) / np.linalg.norm(R))
    assert l2 < MIXED_L2_TOL, l2
    # the mixed path's CFL dt follows the FP64 one to FP32 rounding
    assert abs(g.time - t) <= 1e-5 * t


@pytest.mark.parametrize("name", ["vortex_128x128_p4", "bump_96x32_p3"])
def test_fullsize_2d_autotuned_tiles_match_oracle(oracle, name):
    """The 2D configurations with the stage kernel's tile variant picked by
    the autotuner, as the benchmark runs them (on the 128 x 128 vortex a
    persistent kernel whose blocks walk several tiles): FP64 within 1e-12 of
    the oracle, mixed within 1e-6 relative L2."""
    from fr_learn_b200 import FRG_FP64, FRG_MIXED, Solver

    _, ic, a0, kw, nsteps = _configs()[name]
    mesh, R, dts, t = _oracle_run(oracle, name)
    for prec in (FRG_FP64, FRG_MIXED):
        g = Solver(mesh, precision=prec, **kw)
        g.setInitialCondition(ic, a0)
        v, _ = g.autotune(3)
        assert 0 <= v < g.tile_variant_count()
        gdt = []
        for _ in range(nsteps):
            g.update(1)
            gdt.append(g.dt)
        U = g.get("U_spts")
        if prec == FRG_FP64:
            assert relerr(gdt, dts) < FP64_TOL, v
            assert relerr(U, R) < FP64_TOL, v
            assert abs(g.time - t) <= 1e-12 * t
        else:
            l2 = float(np.linalg.norm(U - R) / np.linalg.norm(R))
            assert l2 < MIXED_L2_TOL, (v, l2)
        g.close()
