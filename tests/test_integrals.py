"""The oracle's output integrals against the reference's own (CPU only).

tests/golden/reference_integrals.npz (made by
tests/golden/make_integrals_golden.py from the FlurryPP sources) holds, for
3D hexahedral cases, the reference's computeWallForce, computeMassFlux
(errorNorm 0, 1, 2) and integrateError (testCase 1, errorNorm 0, 1, 2 at
quadOrder 4) after a few update() steps and one calcResidual(0).  The oracle
runs the same steps (bit-identical to the reference) and must reproduce the
integrals.  The oracle computes the Gauss points of quadOrder by Newton's
method where the reference has a 16-digit table, so the bar is 1e-12 of the
larger of the value's magnitude and 1 (several of these integrals are zero up
to rounding).
"""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "reference_integrals.npz")
PNAMES = ["gamma", "rhoBound", "uBound", "vBound", "wBound", "pBound", "mu_inf", "prandtl", "c_sth",
          "rt_inf", "fixVis", "penFact", "tau", "TWall", "RGas", "uWall", "vWall", "wWall", "dt", "CFL"]
CASES = ["euler_p2_vortex", "euler_p3_freestream", "ns_p2_walls", "ns_p3_sutherland_freestream",
         "advection_p3_gauss", "advection_p2_sine"]
BOX = (-5.0, 5.0, -5.0, 5.0)  # calcError's period for a mesh the reference reads


def close(a, b, tol=1e-12):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return bool(np.all(np.abs(a - b) <= tol * max(float(np.abs(b).max()), 1.0)))


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def integrals_case(golden, name):
    """Mesh, oracle/solver keyword arguments, icType, quadOrder, steps."""
    from fr_learn_b200.mesh import Mesh

    pre = f"{name}/"
    mesh = Mesh(3, golden[pre + "xv"], golden[pre + "c2v"], golden[pre + "bc"])
    order, equation, viscous, icType, quadOrder, nsteps = (int(x) for x in golden[pre + "setup"])
    prm = dict(zip(PNAMES, golden[pre + "params"].tolist()))
    prm["fixVis"] = int(prm["fixVis"])
    dtType = 0 if name in ("euler_p2_vortex", "advection_p3_gauss", "advection_p2_sine") else 1
    kw = dict(nDims=3, order=order, equation=equation, viscous=viscous, dtType=dtType, riemannType=0, **prm)
    return mesh, kw, icType, quadOrder, nsteps


@pytest.mark.parametrize("name", CASES)
def test_oracle_integrals_match_reference(oracle, golden, name):
    mesh, kw, ic, qo, nsteps = integrals_case(golden, name)
    pre = f"{name}/"
    o = oracle.Oracle(oracle.params(**kw), mesh)
    o.set_ic(ic)
    o.update(nsteps)
    assert close(o.U(), golden[pre + "U_spts"], 1e-13)
    assert abs(o.time - float(golden[pre + "time"][0])) <= 1e-13
    o.calc_residual(0)
    assert close(o.wall_force(), golden[pre + "wall_force"])
    for en in range(3):
        assert close(o.mass_flux(en), golden[pre + f"mass_flux_{en}"]), en
    for en in range(3):
        assert close(o.integrate_error(ic, en, qo, BOX), golden[pre + f"error_{en}"]), en
