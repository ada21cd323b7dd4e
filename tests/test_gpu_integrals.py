"""The output integrals on the device (frg_wall_force, frg_mass_flux,
frg_integrate_error) against the oracle, which tests/test_integrals.py pins
to the reference's own computeWallForce / computeMassFlux / integrateError.

FP64: within 1e-12 of the larger of the value's magnitude and 1 (several of
the integrals are zero up to rounding; the device sums in another order).
Mixed mode: the traces are FP32, so within 1e-5 on the same scale.
"""
import numpy as np
import pytest

from conftest import relerr  # noqa: F401
from test_integrals import BOX, CASES, close, integrals_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def golden():
    import os

    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_integrals.npz"))


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", CASES)
def test_device_integrals_match_oracle_3d(oracle, golden, name, precision):
    from fr_learn_b200 import Solver

    mesh, kw, ic, qo, nsteps = integrals_case(golden, name)
    o = oracle.Oracle(oracle.params(**kw), mesh)
    o.set_ic(ic)
    o.update(nsteps)
    o.calc_residual(0)
    kw = {k: v for k, v in kw.items() if k != "nDims"}
    g = Solver(mesh, precision=precision, **kw)
    g.set("U_spts", o.U())
    g.setIter(nsteps, 0)
    tol = 1e-12 if precision == 0 else 1e-5
    assert close(g.computeWallForce(), o.wall_force(), tol)
    for en in range(3):
        assert close(g.computeMassFlux(en), o.mass_flux(en), tol), en
    # integrateError at the oracle's time: the same steps run on the device
    g2 = Solver(mesh, precision=0, **kw)
    g2.setInitialCondition(ic)
    g2.update(nsteps)
    assert abs(g2.time - o.time) <= 1e-13
    for en in range(3):
        assert close(g2.integrateError(ic, en, qo, BOX), o.integrate_error(ic, en, qo, BOX)), en


def _cases_2d():
    from fr_learn_b200 import box2d, bump2d

    c = np.sqrt(1.4)
    return {
        "vortex_periodic_p4": (box2d(8, 8, -10, 10, -10, 10, perturb=0.1, seed=51), 1,
                               dict(order=4, riemannType=1, dtType=1, CFL=0.5), (-10.0, 10.0, -10.0, 10.0)),
        "bump_char_slip_p3": (bump2d(12, 4), 0, dict(order=3, riemannType=1, dtType=1, CFL=0.5, uBound=0.5 * c,
                                                     pBound=1.0), (-5.0, 5.0, -5.0, 5.0)),
        "ns_bump_walls_p2": (bump2d(10, 4, bc_wall="adiabatic_noslip", bc_top="isothermal_noslip"), 0,
                             dict(order=2, riemannType=0, viscous=1, mu_inf=0.01, prandtl=0.72, fixVis=1,
                                  penFact=0.3, tau=1.0, TWall=1.0, RGas=1.0 / 1.4, dtType=1, CFL=0.3,
                                  uBound=0.3 * c, pBound=1.0), (-5.0, 5.0, -5.0, 5.0)),
        "advection_gauss_p3": (box2d(6, 6, perturb=0.1, seed=52), 0, dict(order=3, equation=0, dt=1e-3),
                               (-5.0, 5.0, -5.0, 5.0)),
    }


@pytest.mark.parametrize("name", list(_cases_2d()))
def test_device_integrals_match_oracle_2d(oracle, name):
    from fr_learn_b200 import Solver

    mesh, ic, kw, box = _cases_2d()[name]
    o = oracle.Oracle(oracle.params(nDims=2, **kw), mesh)
    o.set_ic(ic)
    g = Solver(mesh, **kw)
    g.setInitialCondition(ic)
    o.update(3)
    g.update(3)
    o.calc_residual(0)
    assert close(g.computeWallForce(), o.wall_force())
    for en in range(3):
        assert close(g.computeMassFlux(en), o.mass_flux(en)), en
    for en in range(3):
        for qo in (3, 8):
            assert close(g.integrateError(ic, en, qo, box), o.integrate_error(ic, en, qo, box)), (en, qo)
